// Test infrastructure only (oracle/ref_rigid_harness.cu).
// Stand-in for the reference's FixBond.h (FixRigid.h needs only Bond)
#pragma once
#include "Bond.h"
#include "Fix.h"
#include "State.h"
