// Test infrastructure only (oracle/ref_grid_harness.cu).
// Stand-in for the reference's State.h: the members GridGPU.cu reads
#pragma once
#include <algorithm>
#include <cassert>
#include <cstdint>
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
class State {
public:
    bool is2d = false;
    bool requiresCharges = false;
    BoundsGPU boundsGPU;
    DeviceManager devManager;
    std::vector<Fix *> fixes;
    std::vector<Atom> atoms;
    GPUData gpd;
    int64_t turn = 0;
    int nlistBuildCount = 0;
    std::vector<int64_t> nlistBuildTurns;
    int nThreadPerBlock = 256, nThreadPerAtom = 1, nPerRingPoly = 1;
    int maxIdExisting = 0;
};
