// Test infrastructure only (oracle/ref_nh_harness.cu, oracle/ref_berendsen_harness.cu).
// Stand-in for the reference's State.h: the members the barostats read,
// with the reference's types (the time step and the unit factors are real,
// State.h:117, Units.h:8-13)
#pragma once
#include <cstdint>
#include <iostream>
#include <vector>
#include "Atom.h"
#include "BoundsGPU.h"
#include "GPUArrayGlobal.h"
#include "GPUData.h"
class Fix;
enum UNITS { REAL, LJ };
struct Units {
    real boltz = 1.0, nktv_to_press = 1.0, ftm_to_v = 1.0, mvv_to_eng = 1.0;
    int unitType = LJ;
};
class State {
public:
    bool is2d = false;
    BoundsGPU boundsGPU;
    Units units;
    std::vector<Atom> atoms;
    std::vector<Fix *> fixes;
    GPUData gpd;
    int64_t turn = 0, runInit = 0, runningFor = 0;
    real dt = 0.0;
    void findRigidBodies() {}
};
