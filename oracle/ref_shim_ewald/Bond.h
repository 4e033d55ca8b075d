// Test infrastructure only (oracle/ref_ewald_harness.cu).
// Stand-in for the reference's Bond.h: the bond record GridGPU.cu reads
#pragma once
#include <boost/variant.hpp>
struct Bond {
    int ids[2];
};
typedef boost::variant<Bond> BondVariant;
// the visitor that views any bond as a Bond
class bondDowncast : public boost::static_visitor<const Bond &> {
    const BondVariant &bv_;
public:
    explicit bondDowncast(BondVariant &bv) : bv_(bv) {}
    template <class T> const Bond &operator()(const T &) const { return bv_.v; }
};
