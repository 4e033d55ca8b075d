// Harness around the REFERENCE's own SETTLE kernels -- TEST INFRASTRUCTURE
// ONLY.
//
// oracle/ref.mk compiles the reference's src/Fixes/FixRigid.cu where it lies,
// for sm_100a with the reference's nvcc flags, against the stand-in headers
// of oracle/ref_shim_rigid/ (State, Fix, FixBond, Bond and the Boost.Python
// names FixRigid.cu mentions; the split include path makes them shadow the
// reference's own).  The constants of the rigid water (FixRigidData) come
// from the reference's own FixRigid: createRigid for every molecule, then
// setStyleBondLengths, set_fixed_sides and populateRigidData as
// FixRigid::prepareForRun calls them (FixRigid.cu:1740-1765); private members
// are opened to this file only for that.  Every kernel launched here is the
// reference's: compute_COM, save_prev_val, settlePositions, setMSite,
// settleVelocities, with the arguments FixRigid::prepareForRun /
// postNVE_X / postNVE_V give them.  The only code written here is the C entry
// point that lays the sites out (molecule m at 4m .. 4m+3: O, H1, H2, M; id =
// index) in plain device arrays.
#define private public
#include "FixRigid.cu"
#undef private
#include "Atom.cpp"     // Atom::setNDF, which FixRigid::assignNDF calls
#include "pugixml.cpp"  // the XML reader behind Fix::getRestartNode

#include <memory>
#include <vector>

extern "C" {

// mode 1 (a step's first half after the drift, FixRigid::postNVE_X):
//   xs_0 <- x0 (save_prev_val), SETTLE the positions x and velocities v
//   (settlePositions), place M (setMSite); x and v are updated in place.
// mode 2 (the second half after the kick, FixRigid::postNVE_V): settle the
//   velocities v at the positions x (settleVelocities).
// masses: O, H, M.  Returns 0 or a CUDA error code.
int ref_settle(int nmol, const float *x0, float *x, float *v, const double masses[3], const float lo[3],
               const float L[3], double dt, double ftm_to_v, int mode) {
    const int n = 4 * nmol;
    auto st = std::make_shared<State>();
    st->units.ftm_to_v = ftm_to_v;
    st->dt = dt;
    st->boundsGPU = BoundsGPU(make_real3(lo[0], lo[1], lo[2]), make_real3(L[0], L[1], L[2]), make_real3(1, 1, 1));
    st->atoms.reserve(n);
    st->idToIdx.resize(n);
    for (int i = 0; i < n; i++) {
        const int k = i % 4;
        const double m = k == 0 ? masses[0] : (k == 3 ? masses[2] : masses[1]);
        st->atoms.push_back(Atom(Vector(x0[4 * i], x0[4 * i + 1], x0[4 * i + 2]), k == 0 ? 0 : (k == 3 ? 2 : 1), i,
                                 m, 0.0, nullptr));
        st->idToIdx[i] = i;
    }
    FixRigid fix(st, "rigid", "TIP4P/2005");
    for (int mol = 0; mol < nmol; mol++) fix.createRigid(4 * mol, 4 * mol + 1, 4 * mol + 2, 4 * mol + 3);
    fix.nMolecules = nmol;
    fix.fixRigidData = FixRigidData();
    fix.setStyleBondLengths();
    fix.set_fixed_sides();
    fix.populateRigidData();
    const FixRigidData data = fix.fixRigidData;

    std::vector<real4> hx(n), hx0(n), hv(n), hf(n, make_real4(0, 0, 0, 0));
    std::vector<int> hidx(n);
    for (int i = 0; i < n; i++) {
        hx[i] = make_real4(x[4 * i], x[4 * i + 1], x[4 * i + 2], x[4 * i + 3]);
        hx0[i] = make_real4(x0[4 * i], x0[4 * i + 1], x0[4 * i + 2], x0[4 * i + 3]);
        hv[i] = make_real4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
        hidx[i] = i;
    }
    real4 *dx, *dx0, *dv, *df, *dsave, *dcom;
    int4 *dwater;
    int *didx;
    Virial *dvir;
    cudaMalloc(&dx, n * sizeof(real4));
    cudaMalloc(&dx0, n * sizeof(real4));
    cudaMalloc(&dv, n * sizeof(real4));
    cudaMalloc(&df, n * sizeof(real4));
    cudaMalloc(&dsave, 3 * nmol * sizeof(real4));
    cudaMalloc(&dcom, nmol * sizeof(real4));
    cudaMalloc(&dwater, nmol * sizeof(int4));
    cudaMalloc(&didx, n * sizeof(int));
    cudaMalloc(&dvir, n * sizeof(Virial));
    cudaMemcpy(dx, hx.data(), n * sizeof(real4), cudaMemcpyHostToDevice);
    cudaMemcpy(dx0, hx0.data(), n * sizeof(real4), cudaMemcpyHostToDevice);
    cudaMemcpy(dv, hv.data(), n * sizeof(real4), cudaMemcpyHostToDevice);
    cudaMemcpy(df, hf.data(), n * sizeof(real4), cudaMemcpyHostToDevice);
    cudaMemcpy(dwater, fix.waterIds.data(), nmol * sizeof(int4), cudaMemcpyHostToDevice);
    cudaMemcpy(didx, hidx.data(), n * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(dcom, fix.invMassSums.data(), nmol * sizeof(real4), cudaMemcpyHostToDevice);
    cudaMemset(dvir, 0, n * sizeof(Virial));
    const BoundsGPU &bounds = st->boundsGPU;
    const real rdt = (real)dt;
    const real dtf = 0.5f * (real)dt * (real)ftm_to_v;
    const double invdt = 1.0 / dt;
    if (mode == 1) {
        compute_COM<FixRigidData><<<NBLOCK(nmol), PERBLOCK>>>(dwater, dx0, dv, didx, nmol, dcom, bounds, data);
        save_prev_val<<<NBLOCK(nmol), PERBLOCK>>>(dwater, dx0, dsave, nmol, didx);
        settlePositions<FixRigidData, false><<<NBLOCK(nmol), PERBLOCK>>>(dwater, dx, dsave, dv, df, dvir, dcom, data,
                                                                         nmol, rdt, dtf, didx, bounds, 0, invdt,
                                                                         1.0);
        setMSite<FixRigidData><<<NBLOCK(nmol), PERBLOCK>>>(dwater, didx, dx, nmol, bounds, data);
    } else {
        save_prev_val<<<NBLOCK(nmol), PERBLOCK>>>(dwater, dx, dsave, nmol, didx);
        settleVelocities<FixRigidData, false><<<NBLOCK(nmol), PERBLOCK>>>(dwater, dx, dsave, dv, df, dvir, dcom, data,
                                                                          nmol, rdt, dtf, didx, bounds, 0);
    }
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) {
        cudaMemcpy(hx.data(), dx, n * sizeof(real4), cudaMemcpyDeviceToHost);
        cudaMemcpy(hv.data(), dv, n * sizeof(real4), cudaMemcpyDeviceToHost);
        for (int i = 0; i < n; i++) {
            x[4 * i] = hx[i].x; x[4 * i + 1] = hx[i].y; x[4 * i + 2] = hx[i].z;
            v[4 * i] = hv[i].x; v[4 * i + 1] = hv[i].y; v[4 * i + 2] = hv[i].z;
        }
    }
    cudaFree(dx); cudaFree(dx0); cudaFree(dv); cudaFree(df); cudaFree(dsave); cudaFree(dcom);
    cudaFree(dwater); cudaFree(didx); cudaFree(dvir);
    return (int)e;
}

}  // extern "C"
