// Test infrastructure only (oracle/ref_nh_harness.cu, oracle/ref_berendsen_harness.cu).
// Stand-in for <Python.h>: nothing of it is used by the barostat code.
#pragma once
