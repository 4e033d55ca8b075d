// Test infrastructure only (oracle/ref_rigid_harness.cu).
#pragma once
#include <boost/python.hpp>
#include <boost/shared_ptr.hpp>
