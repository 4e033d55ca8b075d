// Harness around the REFERENCE's own Nose-Hoover propagators (the MTK
// barostat's and the particles' chain) -- TEST INFRASTRUCTURE ONLY.
//
// oracle/ref.mk compiles the reference's src/Fixes/FixNoseHoover.cu where it
// lies, with the reference's nvcc flags, against the stand-in headers of
// oracle/ref_shim_nh/ (State, Fix, Mod, Interpolator, the temperature and
// pressure computers, the device arrays and the Boost.Python names
// FixNoseHoover.cu mentions; the split include path makes them shadow the
// reference's own).  The stand-in device arrays hold no device storage, so
// nothing here needs a GPU: the harness calls only host-side code -- the
// four propagators of the isotropic barostat,
//   updateBarostatMasses          (FixNoseHoover.cu:628-667)
//   updateBarostatThermalMasses   (FixNoseHoover.cu:669-700)
//   barostatThermostatIntegrate   (FixNoseHoover.cu:702-793)
//   barostatVelocityIntegrate     (FixNoseHoover.cu:868-943)
// and, for the particles' chain of a thermostat-only fix, prepareFinal,
// updateThermalMasses and thermostatIntegrate -- on a FixNoseHoover whose
// members it sets (private members are opened to this file only for that),
// and none of the fix's kernel launches.  The only code written here is the
// C entry points that copy the barostat and chain state in and out.
#define private public
#include "FixNoseHoover.cu"
#undef private

#include <memory>

extern "C" {

// One call of the propagator `op` on the barostat state:
//   op 0 updateBarostatMasses(step_init)        -> pmass
//   op 1 updateBarostatThermalMasses(step_init) -> ptm, ptf[1..]
//   op 2 barostatThermostatIntegrate(step_init) -> ptv, ptf, pvel
//   op 3 barostatVelocityIntegrate()            -> pvel
// par: natoms, ndf, T (set point, old and new), P (set point), pfreq
// (1 / the barostat time constant), dt, boltz, nktv_to_press, p_inst (the
// scalar instantaneous pressure), t_inst (the scalar temperature), L[3]
// (box lengths).  pvel, pmass: 3 each (x, y, z); ptv, ptf, ptm: `chain`
// each.  Returns 0, or -1 for an unknown op or a chain shorter than 2.
int ref_nh_barostat(int op, int step_init, const double *par, int chain, double *pvel, double *pmass, double *ptv,
                    double *ptf, double *ptm) {
    if (op < 0 || op > 3 || chain < 2) return -1;
    auto st = boost::shared_ptr<State>(new State());
    const int natoms = (int)par[0];
    st->dt = par[5];
    st->units.boltz = par[6];
    st->units.nktv_to_press = par[7];
    st->boundsGPU = BoundsGPU(make_real3(0, 0, 0), make_real3(par[10], par[11], par[12]), make_real3(1, 1, 1));
    st->atoms.assign(natoms, Atom(Vector(0, 0, 0), 0, 0, 1.0, 0.0, nullptr));

    FixNoseHoover fix(st, "nh", "all");
    fix.pressMode = PRESSMODE::ISO;
    fix.barostatting = true;
    fix.boltz = st->units.boltz;  // as prepareFinal sets it (:259), from the float units
    fix.ndf = (size_t)par[1];
    fix.setPointTemperature = fix.oldSetPointTemperature = par[2];
    fix.setPointPressure = fix.oldSetPointPressure = par[3];
    fix.pFrequency = par[4];
    fix.currentPressure = Virial(par[8], par[8], par[8], 0, 0, 0);
    fix.currentTempScalar = par[9];
    fix.pchainLength = (size_t)chain;
    fix.nTimesteps_b = 1;
    fix.n_ys_b = 1;
    fix.weight = std::vector<double>(1, 1.0);
    fix.pFlags = std::vector<bool>{true, true, true, false, false, false};
    fix.pressVel = std::vector<double>(6, 0.0);
    fix.pressMass = std::vector<double>(6, 0.0);
    fix.pressForce = std::vector<double>(6, 0.0);
    for (int i = 0; i < 3; i++) {
        fix.pressVel[i] = pvel[i];
        fix.pressMass[i] = pmass[i];
    }
    fix.pressThermVel.assign(ptv, ptv + chain);
    fix.pressThermForce.assign(ptf, ptf + chain);
    fix.pressThermMass.assign(ptm, ptm + chain);

    const bool si = step_init != 0;
    if (op == 0) fix.updateBarostatMasses(si);
    else if (op == 1) fix.updateBarostatThermalMasses(si);
    else if (op == 2) fix.barostatThermostatIntegrate(si);
    else fix.barostatVelocityIntegrate();

    for (int i = 0; i < 3; i++) {
        pvel[i] = fix.pressVel[i];
        pmass[i] = fix.pressMass[i];
    }
    for (int i = 0; i < chain; i++) {
        ptv[i] = fix.pressThermVel[i];
        ptf[i] = fix.pressThermForce[i];
        ptm[i] = fix.pressThermMass[i];
    }
    return 0;
}

// One call on the particles' Nose-Hoover chain of a thermostat-only fix
// (setTemperature(T, tau), FixNoseHoover.cu:221-225):
//   op 0 prepareFinal (:240-290, thermostatting only) with the kinetic
//        energy *ke (sum m v^2) -> masses, forces, ke
//   op 1 updateThermalMasses (:1034-1041)                -> tmass
//   op 2 thermostatIntegrate(step_init) (:795-866) on *ke -> tvel, tforce,
//        ke, scale (the accumulated velocity factor, *scale in, out)
// par: natoms, ndf, T, tau, dt, boltz.  tvel, tforce, tmass: `chain` each
// (in and out).  The fix keeps the kinetic energy and the scale as floats,
// so *ke and *scale come back float-rounded.  Returns 0, or -1 for an
// unknown op or a chain shorter than 2.
int ref_nh_chain(int op, int step_init, const double *par, int chain, double *tvel, double *tforce, double *tmass,
                 double *ke, double *scale) {
    if (op < 0 || op > 2 || chain < 2) return -1;
    auto st = boost::shared_ptr<State>(new State());
    const int natoms = (int)par[0];
    st->dt = par[4];
    st->units.boltz = par[5];
    st->boundsGPU = BoundsGPU(make_real3(0, 0, 0), make_real3(10, 10, 10), make_real3(1, 1, 1));
    st->atoms.assign(natoms, Atom(Vector(0, 0, 0), 0, 0, 1.0, 0.0, nullptr));

    FixNoseHoover fix(st, "nh", "all");
    fix.setTemperature(par[2], par[3]);
    fix.chainLength = (size_t)chain;
    fix.thermVel.assign(tvel, tvel + chain);
    fix.thermForce.assign(tforce, tforce + chain);
    fix.thermMass.assign(tmass, tmass + chain);
    fix.boltz = st->units.boltz;  // as prepareFinal sets it (:259), from the float units
    fix.ndf = (size_t)par[1];
    fix.setPointTemperature = fix.oldSetPointTemperature = par[2];
    fix.ke_current = (real)*ke;
    fix.scale = make_real3((real)*scale, (real)*scale, (real)*scale);

    if (op == 0) {
        // calculateKineticEnergy reads these from the temperature computer
        fix.tempComputer.ndf = (int64_t)par[1];
        fix.tempComputer.totalKEScalar = *ke;
        fix.tempComputer.tempScalar = *ke / (par[1] * par[5]);
        fix.prepareFinal();
    } else if (op == 1) {
        fix.updateThermalMasses();
    } else {
        fix.thermostatIntegrate(step_init != 0);
    }

    for (int i = 0; i < chain; i++) {
        tvel[i] = fix.thermVel[i];
        tforce[i] = fix.thermForce[i];
        tmass[i] = fix.thermMass[i];
    }
    *ke = fix.ke_current;
    *scale = fix.scale.x;
    return 0;
}

}  // extern "C"
