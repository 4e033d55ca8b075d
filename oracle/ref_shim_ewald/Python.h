// Test infrastructure only (oracle/ref_ewald_harness.cu).
// by the grid kernels the harness compiles.
#pragma once
