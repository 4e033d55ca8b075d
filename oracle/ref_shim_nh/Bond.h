// Test infrastructure only (oracle/ref_nh_harness.cu, oracle/ref_berendsen_harness.cu).
// Stand-in for the reference's Bond.h: the bond record the Fix stand-in names
#pragma once
#include <array>
#include <boost/variant.hpp>
class Bond {
public:
    std::array<int, 2> ids;
    int type;
};
typedef boost::variant<Bond> BondVariant;
