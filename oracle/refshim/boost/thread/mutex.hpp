// Minimal stand-in for <boost/thread/mutex.hpp> (reference-kernel harness only).
#pragma once
#include <mutex>
namespace boost {
struct mutex : std::mutex {
    typedef std::lock_guard<std::mutex> scoped_lock;
};
}
