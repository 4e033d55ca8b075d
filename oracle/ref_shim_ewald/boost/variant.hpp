// Test infrastructure only (oracle/ref_ewald_harness.cu).
// Stand-in for <boost/variant.hpp>: a one-alternative variant, enough for
// GridGPU.cu's exclusion code to compile (no bonds are ever passed to it)
#pragma once
namespace boost {
template <class R> struct static_visitor { typedef R result_type; };
template <class T> struct variant {
    T v;
    variant() {}
    variant(const T &t) : v(t) {}
};
template <class T, class V> T &get(V &v) { return v.v; }
template <class T, class V> const T &get(const V &v) { return v.v; }
template <class Vis, class V> typename Vis::result_type apply_visitor(const Vis &vis, V &v) { return vis(v.v); }
}  // namespace boost
