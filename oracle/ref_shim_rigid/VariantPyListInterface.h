// Test infrastructure only (oracle/ref_rigid_harness.cu).
#pragma once
