// Test infrastructure only (oracle/ref_grid_harness.cu).
// Stand-in for the reference's Fix.h: the two hooks GridGPU.cu calls
#pragma once
#include <vector>
#include "Bond.h"
class Fix {
public:
    virtual ~Fix() {}
    virtual bool handleLocalData() { return true; }
    virtual std::vector<BondVariant> *getBonds() { return nullptr; }
};
