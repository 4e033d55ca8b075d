// Test infrastructure only (oracle/ref_nh_harness.cu, oracle/ref_berendsen_harness.cu).
// Stand-in for the reference's DataComputerTemperature: the fields
// FixNoseHoover.cu reads, set by the harness (the GPU reductions are not
// part of what the harness runs)
#pragma once
#include <cstdint>
#include <string>
#include "Virial.h"
class State;
namespace MD_ENGINE {
class DataComputerTemperature {
public:
    double tempScalar = 0.0, totalKEScalar = 0.0;
    Virial tempTensor;
    int64_t ndf = 0;
    DataComputerTemperature(State *, std::string) {}
    void prepareForRun() {}
    void computeScalar_GPU(bool, uint32_t) {}
    void computeScalar_CPU() {}
    void computeTensor_GPU(bool, uint32_t) {}
    void computeTensor_CPU() {}
    void computeTensorFromScalar() {}
    void computeScalarFromTensor() {}
};
}  // namespace MD_ENGINE
