// Test infrastructure only (oracle/ref_nh_harness.cu, oracle/ref_berendsen_harness.cu).
// Stand-in for the reference's Interpolator: a constant set point (the
// harnesses drive the barostats at a fixed temperature and pressure)
#pragma once
#include <cstdint>
#include <vector>
#include <boost/python.hpp>
class Interpolator {
public:
    double constVal = 0.0, currentVal = 0.0;
    int64_t turnBeginRun = 0, turnFinishRun = 0;
    bool finished = false;
    Interpolator() {}
    explicit Interpolator(double v) : constVal(v), currentVal(v) {}
    explicit Interpolator(boost::python::object) {}
    Interpolator(boost::python::list, boost::python::list) {}
    void computeCurrentVal(int64_t) { currentVal = constVal; }
    double getCurrentVal() { return constVal; }
    void finishRun() {}
};
