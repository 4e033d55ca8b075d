// Harness around the REFERENCE's own P3M splitting-parameter choice -- TEST
// INFRASTRUCTURE ONLY.
//
// oracle/ref.mk compiles the reference's src/Fixes/FixChargeEwald.cu and
// FixCharge.cu where they lie, with the reference's nvcc flags, against the
// stand-in headers of oracle/ref_shim_ewald/ (State, Fix and the Boost.Python
// names; the split include path makes them shadow the reference's own).
// The harness constructs a FixChargeEwald on the CPU and calls its host-side
// FixChargeEwald::find_optimal_parameters (FixChargeEwald.cu:918-967, the
// secant solve of DeltaF_k = DeltaF_real, :865-883) with the mesh, cutoff,
// interpolation order and total squared charge set directly (private members
// are opened to this file only for that): setParameters, which allocates the
// mesh on the device, and every kernel of the fix are left out, so nothing
// here needs a GPU.  The only code written here is the C entry point.
#define private public
#define protected public
#include "FixChargeEwald.cu"
#include "FixCharge.cu"
#include "FixChargePairDSF.cu"  // the DSF fix type name the evaluator picker compares against
#undef protected
#undef private
#include "GridGPU.cu"           // the neighbour grid the stand-in State holds
#include "GPUArrayDevice.cpp"  // the device-array base class the grid's arrays derive from
#include "GPUArrayDeviceGlobal.cu"  // its memset helper
#include "memset_defs.cu"          // and the memset kernels behind it

extern "C" {

// find_optimal_parameters for natoms atoms in a box of sides L, mesh sz,
// real-space cutoff rcut, interpolation order `order`, total squared charge
// q2 (times qqr_to_eng, as setTotalQ2 leaves it).  Out: *alpha (the fix
// keeps it as a float) and *error (the RMS force error estimate
// DeltaF_k + DeltaF_real at it).  Returns 0, or -1 for an order outside 1..7.
int ref_ewald_alpha(int natoms, const double L[3], const int sz[3], double rcut, int order, double q2,
                    double *alpha, double *error) {
    if (order < 1 || order > 7) return -1;
    auto st = boost::shared_ptr<State>(new State());
    st->boundsGPU = BoundsGPU(make_real3(0, 0, 0), make_real3(L[0], L[1], L[2]), make_real3(1, 1, 1));
    st->atoms.assign(natoms, Atom(Vector(0, 0, 0), 0, 0, 1.0, 0.0, nullptr));
    FixChargeEwald fix(st, "ewald", "all");
    fix.sz = make_int3(sz[0], sz[1], sz[2]);
    fix.r_cut = (real)rcut;
    fix.interpolation_order = order;
    fix.total_Q2 = (real)q2;
    *error = fix.find_optimal_parameters(false);
    *alpha = fix.alpha;
    return 0;
}

}  // extern "C"
