// Test infrastructure only (oracle/ref_nh_harness.cu, oracle/ref_berendsen_harness.cu).
// Stand-in for <boost/shared_ptr.hpp>
#pragma once
#include <memory>
namespace boost {
using std::shared_ptr;
}
