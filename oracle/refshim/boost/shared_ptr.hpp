// Minimal stand-in for <boost/shared_ptr.hpp> (reference-kernel harness only).
#pragma once
#include <memory>
namespace boost {
using std::shared_ptr;
}
