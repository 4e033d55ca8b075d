// Harness around the REFERENCE's own Berendsen barostat step -- TEST
// INFRASTRUCTURE ONLY.
//
// oracle/ref.mk compiles the reference's src/Fixes/FixPressureBerendsen.cu
// where it lies, with the reference's nvcc flags, against the stand-in
// headers of oracle/ref_shim_nh/ (the same as oracle/ref_nh_harness.cu's).
// The harness runs the reference's FixPressureBerendsen::stepFinal
// (FixPressureBerendsen.cu:26-46) on the CPU: the stand-in pressure
// computer hands it the instantaneous scalar pressure, the stand-in
// Mod::scaleSystem records the scale factors the step passes on (the
// dilation, after the clamp, as the float the reference's real3 holds).
// The only code written here is the C entry point, and one macro: the
// reference always defines DEBUG (globalDefs.h:7), so its CUT_CHECK_ERROR
// after the rescale synchronizes the device and asserts on the last CUDA
// error, which fails on a machine without a GPU; the stand-in rescale
// launches nothing, so the check is compiled out here.
#include "globalDefs.h"
#undef CUT_CHECK_ERROR
#define CUT_CHECK_ERROR(err) do { } while (false)
#include "FixPressureBerendsen.cu"

extern "C" {

// One Berendsen step: target pressure, instantaneous pressure, period, dt
// (held as the reference's float time step), bulk modulus (< 0: the
// fix's default), maxDilation (< 0: the fix's default).  Out: dilation[3],
// the factors the step scales the box by.  Returns 0.
int ref_berendsen_dilation(double target, double pressure, double period, double dt, double bulk, double max_dil,
                           float *dilation) {
    auto st = boost::shared_ptr<State>(new State());
    st->dt = (real)dt;
    FixPressureBerendsen fix(st, "berendsen", target, period, 1);
    if (bulk >= 0) fix.bulkModulus = bulk;
    if (max_dil >= 0) fix.setParameters(max_dil);
    fix.pressureComputer.pressureScalar = pressure;
    Mod::lastScale() = make_real3(0, 0, 0);
    fix.stepFinal();
    const real3 s = Mod::lastScale();
    dilation[0] = s.x;
    dilation[1] = s.y;
    dilation[2] = s.z;
    return 0;
}

}  // extern "C"
