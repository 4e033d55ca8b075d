"""The oracle's thermostat and barostats against the reference's own, on
CPU: the MTK propagator (oracle/mtk.py vs FixNoseHoover.cu:
updateBarostatMasses :628-667, updateBarostatThermalMasses :669-700,
barostatThermostatIntegrate :702-793, barostatVelocityIntegrate :868-943),
the particles' Nose-Hoover chain (oracle.NoseHooverChain vs prepareFinal
:240-290, thermostatIntegrate :795-866, updateThermalMasses :1034-1041) and
the Berendsen dilation (oracle/berendsen.py vs
FixPressureBerendsen::stepFinal, FixPressureBerendsen.cu:26-46).

tests/golden/ref_barostat.json holds the reference's outputs
(tests/golden/make_ref_barostat.py, from FixNoseHoover.cu compiled from
source); where oracle/_ref/librefbarostat.so is built the reference also runs
live.  In its own precision (float pressure, cell kick, volume and time
step) the oracle reproduces the reference call for call, bit for bit with
this image's libm (the test allows 1e-14 for another libm's exp); in FP64,
the precision the library's propagator computes in, it stays within the
float rounding of those four quantities (relative 1e-6 on the barostat
variables after 25 steps).  The chain likewise: bit for bit in the
reference's precision (float frequency, kinetic energy, velocity scale, time
step and Boltzmann constant), within 1e-5 in FP64 over 40 steps (1e-7 in LJ
units; the float Boltzmann constant of real units moves the chain's
(ke - N k T) by up to 3e-6).  The Berendsen dilation matches the reference's
bit for bit in its precision (a float time step and a float factor) and to
float rounding in FP64, except where the cube root's base is negative: the
reference passes NaN to the box rescale there, the library (and the FP64
oracle) takes the lower clamp."""
import json
import os

import numpy as np
import pytest

from oracle import berendsen as B
from oracle import refkernels as R
from oracle.mtk import MTKLJ

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = json.load(open(os.path.join(HERE, "golden", "ref_barostat.json")))


def calls_of_step(k):
    ke1, p1, ke2, p2 = k
    return [(0, 1, None), (1, 1, None), (2, 1, None), (3, 0, (ke1, p1)), (3, 0, (ke2, p2)),
            (0, 0, None), (1, 0, None), (2, 0, None)]


def bare(c, ref_float):
    m = MTKLJ.__new__(MTKLJ)
    m.T, m.P, m.pfreq = c["T"], c["P"], c["pfreq"]
    m.n, m.ndf, m.pc = c["natoms"], c["ndf"], c["chain"]
    # the reference's time step is a float
    m.dt = float(np.float32(c["dt"])) if ref_float else c["dt"]
    m.L = np.asarray(c["L"], np.float64)
    m.pvel, m.pmass = [0.0] * 3, [0.0] * 3
    m.ptv, m.ptf, m.ptm = [0.0] * m.pc, [0.0] * m.pc, [0.0] * m.pc
    return m


def apply(m, op, si, kp, ref_float):
    if op == 0:
        m.barostat_masses()
    elif op == 1:
        m.barostat_thermal_masses()
    elif op == 2:
        m.barostat_thermostat(bool(si))
    else:
        m.barostat_velocity(kp[0], kp[1], ref_float=ref_float)


def state(m):
    return [np.asarray(a, np.float64) for a in (m.pvel, m.pmass, m.ptv, m.ptf, m.ptm)]


def close(got, want, rtol, atol, what):
    for name, g, w in zip(("pvel", "pmass", "ptv", "ptf", "ptm"), got, want):
        np.testing.assert_allclose(g, np.asarray(w), rtol=rtol, atol=atol, err_msg=f"{what}: {name}")


def replay(c, ref_float, rtol, atol):
    m = bare(c, ref_float)
    m.barostat_masses()
    m.barostat_thermal_masses()
    recs = iter(c["records"])
    for s, k in enumerate(c["kicks"]):
        for op, si, kp in calls_of_step(k):
            apply(m, op, si, kp, ref_float)
            r = next(recs, None) if s < len(c["records"]) // 8 else None
            if r is not None:
                assert (r["step"], r["op"], r["step_init"]) == (s, op, si)
                close(state(m), r["out"], rtol, atol, f"{c['name']} step {s} op {op}")
    close(state(m), c["final"], rtol, atol, f"{c['name']} after {len(c['kicks'])} steps")


@pytest.mark.parametrize("c", FIX["cases"], ids=lambda c: c["name"])
def test_oracle_in_reference_precision_matches_reference(c):
    replay(c, True, 1e-14, 0.0)


@pytest.mark.parametrize("c", FIX["cases"], ids=lambda c: c["name"])
def test_oracle_fp64_within_reference_float_rounding(c):
    replay(c, False, 1e-6, 1e-9)


def test_reference_precision_differs_from_fp64_where_float_rounds():
    """a planted difference, on the CPU: the general box (float volume and
    float dt differ from FP64) moves the FP64 replay off the reference's
    values by more than the in-precision tolerance, so that tolerance is not
    vacuous"""
    c = next(c for c in FIX["cases"] if c["name"] == "lj864_general")
    with pytest.raises(AssertionError):
        replay(c, False, 1e-13, 1e-15)


@pytest.mark.skipif(not R.barostat_available(), reason="oracle/_ref/librefbarostat.so not built")
@pytest.mark.parametrize("c", FIX["cases"], ids=lambda c: c["name"])
def test_live_reference_reproduces_fixture(c):
    """the reference propagator compiled here gives the committed values"""
    z = c["chain"]
    st = (np.zeros(3), np.zeros(3), np.zeros(z), np.zeros(z), np.zeros(z))

    def call(st, op, si, kp):
        ke, p = kp if kp is not None else (0.0, 0.0)
        par = [c["natoms"], c["ndf"], c["T"], c["P"], c["pfreq"], c["dt"], 1.0, 1.0, p, ke / c["ndf"]] + c["L"]
        return R.nh_barostat(op, si, par, *st)

    st = call(st, 0, 0, None)
    st = call(st, 1, 0, None)
    for k in c["kicks"]:
        for op, si, kp in calls_of_step(k):
            st = call(st, op, si, kp)
    close(st, c["final"], 0.0, 0.0, c["name"])


@pytest.mark.skipif(not R.barostat_available(), reason="oracle/_ref/librefbarostat.so not built")
def test_live_reference_rejects_bad_calls():
    z = np.zeros(10)
    par = [100, 297, 1.0, 1.0, 1.0, 0.005, 1.0, 1.0, 1.0, 1.0, 5.0, 5.0, 5.0]
    with pytest.raises(RuntimeError):
        R.nh_barostat(7, 0, par, np.zeros(3), np.zeros(3), z, z, z)
    with pytest.raises(RuntimeError):
        R.nh_barostat(0, 0, par, np.zeros(3), np.zeros(3), z[:1], z[:1], z[:1])


def _bargs(c):
    kw = {}
    if c["bulk"] >= 0:
        kw["bulk"] = c["bulk"]
    if c["max_dil"] >= 0:
        kw["max_dil"] = c["max_dil"]
    return (c["target"], c["pressure"], c["period"], c["dt"]), kw


def test_berendsen_in_reference_precision_matches_reference():
    got = [B.dilation(*a, ref_float=True, **kw) for a, kw in map(_bargs, FIX["berendsen"])]
    want = [c["dilation"][0] for c in FIX["berendsen"]]
    assert all(c["dilation"][0] == c["dilation"][1] == c["dilation"][2] or np.isnan(c["dilation"]).all()
               for c in FIX["berendsen"])
    np.testing.assert_array_equal(np.array(got), np.array(want))
    # the grid reaches both clamps, the inside and the NaN of a negative base
    w = np.array(want)
    assert np.isnan(w).sum() >= 4 and (w[~np.isnan(w)] < 1.0).any() and (w[~np.isnan(w)] > 1.0).any()


def test_berendsen_fp64_matches_reference_but_for_the_negative_base():
    for c in FIX["berendsen"]:
        a, kw = _bargs(c)
        d = B.dilation(*a, **kw)
        want = c["dilation"][0]
        if np.isnan(want):
            # the reference's NaN box; the library compresses at the limit
            assert d == 1.0 - kw.get("max_dil", 1e-5), c
        else:
            assert d == pytest.approx(want, rel=1.2e-7, abs=0.0), c


@pytest.mark.skipif(not R.barostat_available(), reason="oracle/_ref/librefbarostat.so not built")
def test_live_reference_berendsen_reproduces_fixture():
    for c in FIX["berendsen"]:
        d = R.berendsen_dilation(c["target"], c["pressure"], c["period"], c["dt"], c["bulk"], c["max_dil"])
        np.testing.assert_array_equal(d.astype(np.float64), np.array(c["dilation"]))


def _acc(scale, sf, ref_float):
    # the fix's velocity scale is a float3 that `scale *= scaleFactor`
    # multiplies by the float-converted factor
    if ref_float:
        return float(np.float32(scale) * np.float32(sf))
    return scale * sf


def chain_replay(c, ref_float, rtol, atol_frac):
    """the thermostat-only fix's calls (prepareFinal; per step stepInit's
    thermostatIntegrate(true) on the scale stepFinal left, that scale applied
    and reset, then stepFinal's thermostatIntegrate(false) on the step's
    kinetic energy) through the
    oracle's chain, checked against the reference's outputs; atol_frac
    scales each array's absolute tolerance by its largest value"""
    from oracle import oracle as O
    nh = O.NoseHooverChain(c["T"], c["tau"], c["ndf"], c["boltz"], c["dt"], c["chain"], ref_float=ref_float)
    kes = c["kes"]

    def check(scale, want, what):
        got = (nh.vel, nh.force, nh.mass, [nh.ke], [scale])
        for name, g, w in zip(("vel", "force", "mass", "ke", "scale"), got, want):
            w = np.atleast_1d(np.asarray(w, np.float64))
            np.testing.assert_allclose(np.asarray(g, np.float64), w, rtol=rtol,
                                       atol=atol_frac * float(np.abs(w).max()), err_msg=f"{c['name']} {what}: {name}")

    nh.prepare(kes[0])
    recs = list(c["records"])
    check(1.0, recs[0]["out"], "prepare")
    nrec = (len(recs) - 1) // 2
    scale = 1.0
    for s in range(len(kes) - 1):
        # stepInit multiplies the scale stepFinal left, then rescale()
        # applies it and resets it to 1
        scale = _acc(scale, nh.integrate(True), ref_float)
        if s < nrec:
            check(scale, recs[1 + 2 * s]["out"], f"step {s} init")
        nh.ke = float(np.float32(kes[s + 1])) if ref_float else kes[s + 1]
        scale = _acc(1.0, nh.integrate(False), ref_float)
        if s < nrec:
            check(scale, recs[2 + 2 * s]["out"], f"step {s} final")
    check(scale, c["final"], "final")
    nh.update_masses()
    np.testing.assert_allclose(nh.mass, c["masses"], rtol=rtol, err_msg=f"{c['name']}: updateThermalMasses")


@pytest.mark.parametrize("c", FIX["chain"], ids=lambda c: c["name"])
def test_chain_in_reference_precision_matches_reference(c):
    chain_replay(c, True, 1e-14, 0.0)


@pytest.mark.parametrize("c", FIX["chain"], ids=lambda c: c["name"])
def test_chain_fp64_within_reference_float_rounding(c):
    chain_replay(c, False, 1e-5, 1e-5)


@pytest.mark.skipif(not R.barostat_available(), reason="oracle/_ref/librefbarostat.so not built")
@pytest.mark.parametrize("c", FIX["chain"], ids=lambda c: c["name"])
def test_live_reference_chain_reproduces_fixture(c):
    par = [c["natoms"], c["ndf"], c["T"], c["tau"], c["dt"], c["boltz"]]
    z = np.zeros(c["chain"])
    v, f, m, ke, sc = R.nh_chain(0, 0, par, z, z, z, c["kes"][0], 1.0)
    for s in range(len(c["kes"]) - 1):
        v, f, m, ke, sc = R.nh_chain(2, 1, par, v, f, m, ke, sc)
        v, f, m, ke, sc = R.nh_chain(2, 0, par, v, f, m, c["kes"][s + 1], 1.0)
    got = (v, f, m, [ke], [sc])
    for g, w in zip(got, c["final"]):
        np.testing.assert_array_equal(np.asarray(g, np.float64), np.atleast_1d(np.asarray(w, np.float64)))
