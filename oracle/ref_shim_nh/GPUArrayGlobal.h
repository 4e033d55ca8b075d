// Test infrastructure only (oracle/ref_nh_harness.cu, oracle/ref_berendsen_harness.cu).
// Stand-in for the reference's GPUArrayGlobal: a sized host array with no
// device storage, so that FixNoseHoover's constructor (which sizes a
// two-element kinetic-energy array) runs on a machine without a GPU.  The
// harness calls only the host-side barostat propagators, which never touch
// it.
#pragma once
#include <cstddef>
#include <vector>
template <class T>
class GPUArrayGlobal {
public:
    std::vector<T> h_data;
    GPUArrayGlobal() {}
    explicit GPUArrayGlobal(int n) : h_data(n) {}
    size_t size() const { return h_data.size(); }
    T *getDevData() { return nullptr; }
    void dataToDevice() {}
    void dataToHost() {}
    void memsetByVal(const T &v) { h_data.assign(h_data.size(), v); }
};
