// Test infrastructure only (oracle/ref_ewald_harness.cu).
// Stand-in for <boost/python.hpp>: the names the barostat sources mention, doing nothing
#pragma once
#include <string>
namespace boost {
struct noncopyable {};
namespace python {
struct no_init_t {};
static no_init_t no_init;
struct object {
    object() {}
    template <class T> object(const T &) {}
};
struct list {
    template <class T> void append(const T &) {}
    template <class T> list &operator[](const T &) { return *this; }
    template <class T> list &operator=(const T &) { return *this; }
};
template <class... T> struct bases {};
template <class... T> struct init {
    template <class... A> init(A &&...) {}
};
struct arg_ {
    template <class T> arg_ &operator=(const T &) { return *this; }
};
inline arg_ arg(const char *) { return arg_(); }
template <class... A> arg_ args(A &&...) { return arg_(); }
inline arg_ operator,(arg_ a, arg_) { return a; }
template <class T, class X = void, class Y = void, class Z = void>
struct class_ {
    template <class... A> class_ &def_readonly_(A &&...) { return *this; }
    template <class... A> class_(A &&...) {}
    template <class... A> class_ &def(A &&...) { return *this; }
    template <class... A> class_ &def_readwrite(A &&...) { return *this; }
    template <class... A> class_ &def_readonly(A &&...) { return *this; }
    template <class... A> class_ &add_property(A &&...) { return *this; }
};
}  // namespace python
}  // namespace boost
