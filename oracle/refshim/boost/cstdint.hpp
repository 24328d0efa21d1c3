// Minimal stand-in for <boost/cstdint.hpp>, only to compile the reference's
// kernel sources for the reference-kernel harness (test infrastructure).
#pragma once
#include <cstdint>
#include <stdint.h>
namespace boost {
using std::int64_t;
using std::uint32_t;
using std::uintmax_t;
}
