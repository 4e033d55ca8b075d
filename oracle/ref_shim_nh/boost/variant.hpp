// Test infrastructure only (oracle/ref_nh_harness.cu, oracle/ref_berendsen_harness.cu).
// Stand-in for <boost/variant.hpp>: a one-alternative variant
#pragma once
namespace boost {
template <class R> struct static_visitor { typedef R result_type; };
template <class T> struct variant {
    T v;
    variant() {}
    variant(const T &t) : v(t) {}
};
template <class T, class V> T &get(V &v) { return v.v; }
}  // namespace boost
