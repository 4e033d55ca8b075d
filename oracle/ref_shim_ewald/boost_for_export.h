// Test infrastructure only (oracle/ref_ewald_harness.cu).
// Stand-in for the reference's boost_for_export.h: the Boost.Python names
// of the stand-in <boost/python.hpp> only
#pragma once
#include <boost/python.hpp>
#include <boost/shared_ptr.hpp>
