// Test infrastructure only (oracle/ref_rigid_harness.cu).
// Stand-in for the reference's State.h: the members FixRigid.cu reads
#pragma once
#include <algorithm>
#include <cassert>
#include <cstdint>
#include <iostream>
#include <vector>
#include <boost/lexical_cast.hpp>
#include "Atom.h"
#include "BoundsGPU.h"
#include "GPUArrayGlobal.h"
#include "GPUData.h"
struct DeviceManager {
    cudaDeviceProp prop;
};
struct DataManager {
    int mode = 0;
    int getVirialModeForTurn(int64_t) { return mode; }
};
enum UNITS { REAL, LJ };
struct Units {
    double ftm_to_v = 0.0;
    int unitType = REAL;
};
class State {
public:
    BoundsGPU boundsGPU;
    DeviceManager devManager;
    DataManager dataManager;
    Units units;
    std::vector<Atom> atoms;
    std::vector<int> idToIdx;
    GPUData gpd;
    int64_t turn = 0;
    double dt = 0.0;
    bool rigidBodies = false;
    bool masslessSites = false;
    Atom &idToAtom(int id) { return atoms[idToIdx[id]]; }
};
