// Test infrastructure only (oracle/ref_ewald_harness.cu).
// Stand-in for the reference's State.h: the members FixChargeEwald.cu and
// FixCharge.cu read, with the reference's types (State.h, Units.h)
#pragma once
#include <algorithm>
#include <cassert>
#include <cstdint>
#include <functional>
#include <vector>
#include "Atom.h"
#include "BoundsGPU.h"
#include "GPUData.h"
#include "GridGPU.h"
class Fix;
enum EXCLUSIONMODE { FORCER, DISTANCE };
struct DeviceManager {
    cudaDeviceProp prop;
};
struct Units {
    real boltz = 1.0, qqr_to_eng = 1.0, mvv_to_eng = 1.0, nktv_to_press = 1.0, ftm_to_v = 1.0;
};
class State {
public:
    bool is2d = false;
    bool requiresCharges = false;
    BoundsGPU boundsGPU;
    struct {
        Vector rectComponents;
    } bounds;  // the CPU box, read by setGridToErrorTolerance only
    GridGPU gridGPU;
    real specialNeighborCoefs[3] = {0, 0, 0};
    DeviceManager devManager;
    Units units;
    std::vector<Fix *> fixes;
    std::vector<Atom> atoms;
    GPUData gpd;
    int64_t turn = 0;
    int nlistBuildCount = 0;
    std::vector<int64_t> nlistBuildTurns;
    int nThreadPerBlock = 256, nThreadPerAtom = 1, nPerRingPoly = 1;
    int maxIdExisting = 0;
    real rCut = 0, dt = 0;
};
