// Test infrastructure only (oracle/ref_nh_harness.cu, oracle/ref_berendsen_harness.cu).
// Stand-in for the reference's DataComputerPressure: the fields
// the barostats read, set by the harnesses
#pragma once
#include <cstdint>
#include <string>
#include "Virial.h"
class State;
namespace MD_ENGINE {
class DataComputerPressure {
public:
    double tempScalar = 0.0, pressureScalar = 0.0;
    Virial tempTensor, pressureTensor;
    int64_t tempNDF = 0;
    bool usingExternalTemperature = false;
    DataComputerPressure(State *, std::string) {}
    void prepareForRun() {}
    void computeScalar_GPU(bool, uint32_t) {}
    void computeScalar_CPU() {}
    void computeTensor_GPU(bool, uint32_t) {}
    void computeTensor_CPU() {}
};
}  // namespace MD_ENGINE
