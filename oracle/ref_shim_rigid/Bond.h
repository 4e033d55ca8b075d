// Test infrastructure only (oracle/ref_rigid_harness.cu).
// Stand-in for the reference's Bond.h: the bond record FixRigid.cu builds
#pragma once
#include <array>
#include <boost/variant.hpp>
class Bond {
public:
    std::array<int, 2> ids;
    int type;
};
typedef boost::variant<Bond> BondVariant;
