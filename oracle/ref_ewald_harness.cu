// Harness around the REFERENCE's own P3M splitting-parameter choice and
// influence function -- TEST INFRASTRUCTURE ONLY.
//
// oracle/ref.mk compiles the reference's src/Fixes/FixChargeEwald.cu and
// FixCharge.cu where they lie, with the reference's nvcc flags, against the
// stand-in headers of oracle/ref_shim_ewald/ (State, Fix and the Boost.Python
// names; the split include path makes them shadow the reference's own).
// The harness constructs a FixChargeEwald and calls, first, its host-side
// FixChargeEwald::find_optimal_parameters (FixChargeEwald.cu:918-967, the
// secant solve of DeltaF_k = DeltaF_real, :865-883) with the mesh, cutoff,
// interpolation order and total squared charge set directly (private members
// are opened to this file only for that; setParameters, which allocates the
// mesh on the device, is not called there); second, setParameters and
// calc_Green_function, whose Green_function_cu kernel computes the influence
// function on the device.  The fix's default-constructed device arrays
// initialise the CUDA runtime, so both run where a GPU is.  The only code
// written here is the C entry points.
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

// The reference's influence function on the device: setParameters (the
// mesh buffers, FixChargeEwald.cu:969-1022), then calc_Green_function
// (:1097-1123, the Green_function_cu kernel, :314-366) for the box of sides
// L, mesh sz (each a power of two from 32 to 1024), splitting parameter
// alpha, interpolation order `order`, with the mesh spacings as
// find_optimal_parameters leaves them (L / sz).  Out: green[sz.x*sz.y*sz.z]
// in the kernel's (x, y, z) order.  Returns 0, a CUDA error code, or -1 for
// an order outside 1..7.
int ref_ewald_green(const double L[3], const int sz[3], double alpha, int order, float *green) {
    if (order < 1 || order > 7) return -1;
    auto st = boost::shared_ptr<State>(new State());
    st->boundsGPU = BoundsGPU(make_real3(0, 0, 0), make_real3(L[0], L[1], L[2]), make_real3(1, 1, 1));
    FixChargeEwald fix(st, "ewald", "all");
    fix.setParameters(sz[0], sz[1], sz[2], (real)9.0, order);
    fix.L = st->boundsGPU.trace();
    fix.h = make_real3(fix.L.x / sz[0], fix.L.y / sz[1], fix.L.z / sz[2]);
    fix.alpha = (real)alpha;
    fix.calc_Green_function();
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return (int)e;
    fix.Green_function.dataToHost();
    const size_t n = (size_t)sz[0] * sz[1] * sz[2];
    for (size_t i = 0; i < n; i++) green[i] = fix.Green_function.h_data[i];
    return 0;
}

}  // extern "C"
