// Test infrastructure only (oracle/ref_rigid_harness.cu, oracle/ref_nh_harness.cu).
#pragma once
#include <boost/python.hpp>
