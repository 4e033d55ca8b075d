"""Generate tests/golden/ref_barostat.json from the reference's own isotropic
MTK barostat propagator (FixNoseHoover.cu: updateBarostatMasses :628-667,
updateBarostatThermalMasses :669-700, barostatThermostatIntegrate :702-793,
barostatVelocityIntegrate :868-943), particle Nose-Hoover chain
(prepareFinal :240-290, thermostatIntegrate :795-866, updateThermalMasses
:1034-1041) and Berendsen step
(FixPressureBerendsen::stepFinal, FixPressureBerendsen.cu:26-46), compiled
from the reference source by oracle/ref.mk into oracle/_ref/librefbarostat.so
(host code; no GPU needed).

Each case drives the barostat variables through the calls one NPT step
makes, in the order of the step's hooks (stepInit: masses, thermal masses,
the barostat chain at the old set point, the first cell-velocity kick;
postNVE_V: the second kick; stepFinal: masses, thermal masses, the chain),
with a seeded kinetic energy and pressure for every kick standing in for
the particles.  The fixture holds the inputs, every call's output for the
first steps and the state after the last.

Run in a checkout where the reference source is present:
    make -f oracle/ref.mk && python tests/golden/make_ref_barostat.py"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import refkernels as R  # noqa: E402

# (name, natoms, ndf, T, P, pfreq, dt, L, chain, steps, recorded steps)
CASES = [
    # box lengths and time step exactly representable in float: the
    # reference's float cell volume and float time step equal the FP64 ones
    ("lj500_chain10", 500, 1497, 1.2, 0.8, 1.0, float(np.float32(0.005)), (8.5, 8.5, 8.5), 10, 25, 3),
    ("lj256_chain4", 256, 765, 0.9, 1.5, 2.0, 0.00390625, (7.0, 7.25, 6.5), 4, 25, 3),
    # general box lengths and dt = 0.005 (the reference rounds both to float)
    ("lj864_general", 864, 2589, 1.1, 0.6, 1.0, 0.005, (10.1, 9.7, 10.3), 10, 25, 0),
]


def calls_of_step(ke1, p1, ke2, p2):
    return [(0, 1, None), (1, 1, None), (2, 1, None), (3, 0, (ke1, p1)), (3, 0, (ke2, p2)),
            (0, 0, None), (1, 0, None), (2, 0, None)]


def run(case):
    name, natoms, ndf, T, P, pfreq, dt, L, chain, steps, rec = case
    rng = np.random.default_rng(20261204 + natoms)
    kicks = []
    for _ in range(steps):
        ke = ndf * T * (1.0 + 0.15 * rng.standard_normal(2))
        p = P + 0.6 * rng.standard_normal(2)
        kicks.append([float(ke[0]), float(p[0]), float(ke[1]), float(p[1])])
    st = (np.zeros(3), np.zeros(3), np.zeros(chain), np.zeros(chain), np.zeros(chain))

    def call(st, op, si, kp):
        ke, p = kp if kp is not None else (0.0, 0.0)
        par = [natoms, ndf, T, P, pfreq, dt, 1.0, 1.0, p, ke / ndf, L[0], L[1], L[2]]
        return R.nh_barostat(op, si, par, *st)

    # the prepare-time masses (FixNoseHoover::prepareFinal)
    st = call(st, 0, 0, None)
    st = call(st, 1, 0, None)
    records = []
    for s, (ke1, p1, ke2, p2) in enumerate(kicks):
        for op, si, kp in calls_of_step(ke1, p1, ke2, p2):
            st = call(st, op, si, kp)
            if s < rec:
                records.append({"step": s, "op": op, "step_init": si, "out": [a.tolist() for a in st]})
    return {"name": name, "natoms": natoms, "ndf": ndf, "T": T, "P": P, "pfreq": pfreq, "dt": dt, "L": list(L),
            "chain": chain, "kicks": kicks, "records": records, "final": [a.tolist() for a in st]}


def berendsen_cases():
    """a grid over the pressure offset (inside the clamp, at both clamps,
    and a negative cube-root base), the period, dt, the bulk modulus and
    maxDilation (-1: the fix's defaults)"""
    out = []
    for target, bulk, max_dil in ((1.0, -1.0, -1.0), (1.0, 20.0, 1e-3), (0.5, 5.0, 2e-2), (3.0, 100.0, 1e-1)):
        for off in (0.0, 1e-4, -1e-4, 0.01, -0.01, 0.3, -0.3, 2.0, -2.0, 40.0, -40.0, 5e3, -5e3):
            for period, dt in ((0.5, 0.005), (2.0, 0.002), (1.0, 0.00390625)):
                p = target - off
                d = R.berendsen_dilation(target, p, period, dt, bulk, max_dil)
                out.append({"target": target, "pressure": p, "period": period, "dt": dt, "bulk": bulk,
                            "max_dil": max_dil, "dilation": [float(x) for x in d]})
    return out


# (name, natoms, ndf, T, tau, dt, boltz, chain, steps, recorded steps)
CHAIN_CASES = [
    ("lj500_chain10", 500, 1497, 1.2, 0.5, 0.005, 1.0, 10, 40, 3),
    ("lj256_chain3", 256, 765, 0.9, 0.1, 0.002, 1.0, 3, 40, 3),
    # rigid TIP4P/2005 in real units (6 per molecule less the centre of mass)
    ("water4096_real", 16384, 24573, 298.0, 100.0, 1.0, 0.0019872067, 10, 40, 0),
]


def run_chain(case):
    """the thermostat-only fix's calls over `steps` steps: prepareFinal on a
    seeded kinetic energy; then per step stepInit's thermostatIntegrate(true)
    (its scale applied and reset by rescale) and stepFinal's
    thermostatIntegrate(false) on the step's seeded kinetic energy"""
    name, natoms, ndf, T, tau, dt, boltz, chain, steps, rec = case
    rng = np.random.default_rng(20261205 + natoms)
    kes = [float(ndf * boltz * T * (1.0 + 0.2 * x)) for x in rng.standard_normal(steps + 1)]
    par = [natoms, ndf, T, tau, dt, boltz]
    z = np.zeros(chain)
    v, f, m, ke, sc = R.nh_chain(0, 0, par, z, z, z, kes[0], 1.0)
    records = [{"step": -1, "op": 0, "step_init": 0, "out": [v.tolist(), f.tolist(), m.tolist(), ke, sc]}]
    for s_ in range(steps):
        v, f, m, ke, sc = R.nh_chain(2, 1, par, v, f, m, ke, sc)
        if s_ < rec:
            records.append({"step": s_, "op": 2, "step_init": 1, "out": [v.tolist(), f.tolist(), m.tolist(), ke, sc]})
        sc = 1.0  # rescale() applies the scale and resets it
        v, f, m, ke, sc = R.nh_chain(2, 0, par, v, f, m, kes[s_ + 1], sc)
        if s_ < rec:
            records.append({"step": s_, "op": 2, "step_init": 0, "out": [v.tolist(), f.tolist(), m.tolist(), ke, sc]})
    # updateThermalMasses on the final state
    v, f, m2, ke, sc = R.nh_chain(1, 0, par, v, f, np.zeros(chain), ke, sc)
    return {"name": name, "natoms": natoms, "ndf": ndf, "T": T, "tau": tau, "dt": dt, "boltz": boltz,
            "chain": chain, "kes": kes, "records": records, "final": [v.tolist(), f.tolist(), m.tolist(), ke, sc],
            "masses": m2.tolist()}


def main():
    if not R.barostat_available():
        raise SystemExit("oracle/_ref/librefbarostat.so is not built")
    out = {"source": "FixNoseHoover.cu barostat propagators and particle chain, FixPressureBerendsen.cu's step, "
                     "compiled from the reference source",
           "cases": [run(c) for c in CASES], "chain": [run_chain(c) for c in CHAIN_CASES],
           "berendsen": berendsen_cases()}
    with open(os.path.join(HERE, "ref_barostat.json"), "w") as f:
        json.dump(out, f, indent=0)
        f.write("\n")


if __name__ == "__main__":
    main()
