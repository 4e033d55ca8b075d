// Test infrastructure only (oracle/ref_grid_harness.cu).
// Stand-in for <boost/python.hpp>: the names GridGPU.cu uses, doing nothing
#pragma once
namespace boost {
struct noncopyable {};
namespace python {
struct no_init_t {};
static no_init_t no_init;
struct list {
    template <class T> void append(const T &) {}
    template <class T> list &operator[](const T &) { return *this; }
    template <class T> list &operator=(const T &) { return *this; }
};
struct arg_ {
    template <class T> arg_ &operator=(const T &) { return *this; }
};
inline arg_ arg(const char *) { return arg_(); }
inline arg_ operator,(arg_ a, arg_) { return a; }
template <class T, class X = void>
struct class_ {
    template <class... A> class_(A &&...) {}
    template <class... A> class_ &def(A &&...) { return *this; }
};
}  // namespace python
}  // namespace boost
