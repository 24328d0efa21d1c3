// Minimal stand-in for <boost/shared_array.hpp> (reference-kernel harness only).
#pragma once
#include <memory>
namespace boost {
template <class T>
using shared_array = std::shared_ptr<T[]>;
}
