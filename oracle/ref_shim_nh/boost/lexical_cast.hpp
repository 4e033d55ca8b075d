// Test infrastructure only (oracle/ref_nh_harness.cu, oracle/ref_berendsen_harness.cu).
// Stand-in for <boost/lexical_cast.hpp> (used only on restart files, which
// the harness never reads)
#pragma once
#include <sstream>
#include <string>
namespace boost {
template <class T, class S> T lexical_cast(const S &s) {
    std::stringstream ss;
    ss << s;
    T t{};
    ss >> t;
    return t;
}
}  // namespace boost
