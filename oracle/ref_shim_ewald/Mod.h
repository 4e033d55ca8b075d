// Test infrastructure only (oracle/ref_ewald_harness.cu).
// Stand-in for the reference's Mod.h (GridGPU.cu calls none of it)
#pragma once
