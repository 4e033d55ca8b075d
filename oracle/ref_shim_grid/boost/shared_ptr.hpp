// Minimal stand-in for <boost/shared_ptr.hpp> so that the reference's
// header-only kernels compile here without Boost (test infrastructure only).
#pragma once
#include <functional>
#include <memory>
namespace boost {
using std::shared_ptr;
}
