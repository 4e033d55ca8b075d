// Test infrastructure only (oracle/ref_rigid_harness.cu).
// Stand-in for <Python.h>: nothing of it is used by the SETTLE code.
#pragma once
