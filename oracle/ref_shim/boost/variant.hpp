// Minimal stand-in for <boost/variant.hpp> (only its name is needed by the
// reference headers the harness includes; test infrastructure only).
#pragma once
#include <cassert>
namespace boost {
template <class T, class V>
T &get(V &v) { return *static_cast<T *>(nullptr); }
}
