// Test infrastructure only (oracle/ref_ewald_harness.cu).
#pragma once
#include <boost/python.hpp>
