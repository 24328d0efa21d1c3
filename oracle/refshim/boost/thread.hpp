// Minimal stand-in for <boost/thread.hpp> (reference-kernel harness only).
#pragma once
#include "thread/mutex.hpp"
#include "shared_ptr.hpp"
