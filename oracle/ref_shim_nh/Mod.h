// Test infrastructure only (oracle/ref_nh_harness.cu, oracle/ref_berendsen_harness.cu).
// Stand-in for the reference's Mod.h: the one call the barostats make (the
// box rescale), which here records the scale factors it is given instead of
// moving the atoms
#pragma once
#include <cstdint>
#include "globalDefs.h"
class State;
namespace Mod {
inline real3 &lastScale() {
    static real3 s = make_real3(0, 0, 0);
    return s;
}
inline void scaleSystem(State *, real3 scaleBy, uint32_t = 1) { lastScale() = scaleBy; }
}  // namespace Mod
