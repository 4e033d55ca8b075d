// Test infrastructure only (oracle/ref_nh_harness.cu, oracle/ref_berendsen_harness.cu).
// Stand-in for the reference's GPUData: the velocity and force arrays
// FixNoseHoover.cu names in its rescaling launches, without device storage
// (the harness runs none of those launches)
#pragma once
#include "GPUArrayGlobal.h"
#include "globalDefs.h"
class GPUData {
public:
    GPUArrayGlobal<real4> vs, fs;
};
