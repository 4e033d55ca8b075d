// Test infrastructure only (oracle/ref_ewald_harness.cu).
// Stand-in for <boost/shared_ptr.hpp>
#pragma once
#include <memory>
namespace boost {
using std::shared_ptr;
}
