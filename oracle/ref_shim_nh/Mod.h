// Test infrastructure only (oracle/ref_nh_harness.cu).
// Stand-in for the reference's Mod.h: the one call FixNoseHoover.cu makes
// (the volume rescale, which the harness does not run)
#pragma once
#include <cstdint>
#include "globalDefs.h"
class State;
namespace Mod {
inline void scaleSystem(State *, real3, uint32_t) {}
}
