"""Pressure control: Mod::scaleSystem and FixPressureBerendsen
(src/Fixes/FixPressureBerendsen.cu).  A box change must carry the positions
(free atoms about the box centre, rigid molecules by their centres of mass),
the P3M Green function and splitting, and the neighbour grids with it: after
it the forces match the FP64 oracle evaluated in the new box.  The barostat's
dilation follows the reference's formula from the pressure it read, and over
a run it drives the pressure of an LJ fluid toward its target."""
import numpy as np
import pytest

from md_engine_b200 import FixNoseHoover, FixPressureBerendsen, IntegratorVerlet, systems
from oracle import berendsen
from tests.helpers import FORCE_RTOL, force_err, oracle_lj_params, oracle_water_params, water_bonds, water_small

pytestmark = pytest.mark.gpu


def _box(st):
    return np.array(st.bounds.lo.v), np.array(st.bounds.hi.v)


def _min_image(d, L):
    return d - L * np.rint(d / L)


def _water_com(x, mol, L, mO=15.9994, mH=1.008):
    o = x[mol[:, 0]]
    d1 = _min_image(x[mol[:, 1]] - o, L)
    d2 = _min_image(x[mol[:, 2]] - o, L)
    return o + (d1 + d2) * (mH / (mO + 2 * mH))


def _water_forces_vs_oracle(oracle, st, sysd, lo, L, rc=6.5, pad=1.0, grid=32, alpha=0.35):
    st.computeForces()
    x, _, fg = st.getAtoms()
    excl = oracle.exclusions_from_bonds(len(x), water_bonds(sysd.molecules))
    xs4 = np.zeros((len(x), 4), np.float32)
    xs4[:, :3] = x
    oracle.wrap_f32(xs4, lo, L)
    cut = np.float32(float(np.float32(rc)) + pad)
    c, nb = oracle.nlist_cells(xs4, lo, L, cut, ids=np.arange(len(x)), excl=excl)
    pr = oracle.pair_forces(x, sysd.types, sysd.q, oracle_water_params(oracle, rc), L, c, nb, qrc=rc, alpha=alpha,
                            qqr_to_eng=oracle.REAL_UNITS["qqr_to_eng"])
    frec = oracle.p3m_forces(x, sysd.q, lo, L, (grid,) * 3, alpha)
    return force_err(fg, pr["f"] + frec)


@pytest.mark.parametrize("form", [1, 2])
@pytest.mark.parametrize("scale", [1.012, 0.992])
def test_scale_system_water_moves_molecules_and_forces_follow(oracle, form, scale):
    sysd = water_small(seed=31)
    st, fx = systems.build_water_state(sysd, rcut=6.5, skin=1.0, grid=32, alpha=0.35, thermostat=False)
    st.pairForm = form
    st.prepare()
    x0, _, _ = st.getAtoms()
    lo0, hi0 = _box(st)
    L0 = hi0 - lo0
    c = 0.5 * (lo0 + hi0)
    st.scaleSystem(scale)
    lo1, hi1 = _box(st)
    L1 = hi1 - lo1
    np.testing.assert_allclose(L1, L0 * scale, rtol=1e-14)
    np.testing.assert_allclose(0.5 * (lo1 + hi1), c, rtol=0, atol=1e-12)
    x1, _, _ = st.getAtoms()
    mol = np.asarray(sysd.molecules)
    com0 = _water_com(x0, mol, L0)
    shift = (c + (com0 - c) * scale) - com0
    for k in range(4):
        d = _min_image(x1[mol[:, k]] - (x0[mol[:, k]] + shift), L1)
        assert np.abs(d).max() < 2e-5, np.abs(d).max()
    # rigid geometry kept
    for a, b in ((0, 1), (0, 2), (1, 2)):
        r0 = np.linalg.norm(_min_image(x0[mol[:, a]] - x0[mol[:, b]], L0), axis=1)
        r1 = np.linalg.norm(_min_image(x1[mol[:, a]] - x1[mol[:, b]], L1), axis=1)
        assert np.abs(r1 - r0).max() < 1e-5
    sysd1 = systems.System(**{**sysd.__dict__, "lo": lo1, "L": L1})
    rel, rms = _water_forces_vs_oracle(oracle, st, sysd1, lo1, L1)
    assert rel < FORCE_RTOL, f"forces after the box change: {rel:.3e} of RMS {rms:.3e}"
    assert st.status()[0] == 0


def test_scale_system_lj_scales_atoms_about_the_centre(oracle):
    sysd = systems.lj_fcc(ncell=12, jitter=0.05, seed=7)
    st, _ = systems.build_lj_state(sysd, rcut=2.5, skin=0.3)
    st.prepare()
    x0, _, _ = st.getAtoms()
    lo0, hi0 = _box(st)
    c = 0.5 * (lo0 + hi0)
    st.scaleSystem(1.03)
    lo1, hi1 = _box(st)
    L1 = hi1 - lo1
    x1, _, _ = st.getAtoms()
    d = _min_image(x1 - (c + (x0 - c) * 1.03), L1)
    assert np.abs(d).max() < 2e-5
    st.computeForces(virialMode=1)
    x, _, fg = st.getAtoms()
    xs4 = np.zeros((len(x), 4), np.float32)
    xs4[:, :3] = x
    oracle.wrap_f32(xs4, lo1, L1)
    cn, nb = oracle.nlist_cells(xs4, lo1, L1, np.float32(2.8), ids=np.arange(len(x)))
    ref = oracle.pair_forces(x, sysd.types, sysd.q, oracle_lj_params(oracle, sysd, 2.5), L1, cn, nb)
    rel, rms = force_err(fg, ref["f"])
    assert rel < FORCE_RTOL


def test_berendsen_dilation_follows_the_reference_formula():
    sysd = systems.lj_fcc(ncell=10, jitter=0.05, seed=9, T=1.5)
    st, _ = systems.build_lj_state(sysd, rcut=2.5, skin=0.3, T=1.5, tau=0.5)
    st.prepare()
    p0, _ = st.pressure()
    baro = FixPressureBerendsen(st, "baro", p0 + 3.0, 0.5, 5)
    baro.setParameters(maxDilation=1e-3)
    baro.bulkModulus = 20.0
    st.activateFix(baro)
    lo0, hi0 = _box(st)
    IntegratorVerlet(st).run(1)  # the barostat fires after the step of turn 0
    assert baro.applications == 1
    p, dil = baro.lastPressure, baro.lastDilation
    # the oracle's FP64 dilation (pinned against the reference's stepFinal)
    want = berendsen.dilation(p0 + 3.0, p, 0.5, 0.005, bulk=20.0, max_dil=1e-3)
    assert dil == pytest.approx(want, rel=1e-15, abs=1e-15)
    assert dil < 1.0  # a target above the pressure compresses
    lo1, hi1 = _box(st)
    np.testing.assert_allclose(hi1 - lo1, (hi0 - lo0) * dil, rtol=1e-14)
    # clamped at maxDilation when the pressure is far off
    baro.pressure = p + 1e4
    IntegratorVerlet(st).run(5)
    assert baro.applications == 2 and baro.lastDilation == pytest.approx(1 - 1e-3, rel=1e-15)


def test_berendsen_drives_lj_pressure_to_target():
    """LJ fluid at T = 1.5: the target pressure 2 above the start is reached
    (mean over the last stretch within a quarter of the initial offset), and
    the box shrinks on the way"""
    sysd = systems.lj_fcc(ncell=10, rho=0.7, jitter=0.05, seed=13, T=1.5)
    st, _ = systems.build_lj_state(sysd, rcut=2.5, skin=0.3, T=1.5, tau=0.5)
    st.prepare()
    IntegratorVerlet(st).run(400)
    p0 = np.mean([st.pressure()[0] for _ in range(1)])
    target = p0 + 2.0
    baro = FixPressureBerendsen(st, "baro", target, 0.5, 1)
    baro.setParameters(maxDilation=2e-3)
    baro.bulkModulus = 20.0
    st.activateFix(baro)
    lo0, hi0 = _box(st)
    it = IntegratorVerlet(st)
    it.run(1500)
    ps = []
    for _ in range(30):
        it.run(10)
        ps.append(baro.lastPressure)
    lo1, hi1 = _box(st)
    assert np.prod(hi1 - lo1) < np.prod(hi0 - lo0)
    assert abs(np.mean(ps) - target) < 0.25 * abs(target - p0), (p0, target, np.mean(ps))
    assert st.status()[0] == 0


def test_berendsen_water_runs_in_the_molecule_form(oracle):
    """rigid TIP4P/2005 under the barostat in the molecule form: the box
    moves every 10 steps, the run stays sound, and the forces in the final
    box match the oracle"""
    sysd = water_small(seed=33)
    st, fx = systems.build_water_state(sysd, rcut=6.5, skin=1.0, grid=32, alpha=0.35, T=298.0, tau=100.0)
    baro = FixPressureBerendsen(st, "baro", 1.0, 1000.0, 10)
    baro.setParameters(maxDilation=1e-3)
    st.activateFix(baro)
    st.prepare()
    assert int(st.pairForm) == 2
    lo0, hi0 = _box(st)
    IntegratorVerlet(st).run(200)
    assert baro.applications == 20
    lo1, hi1 = _box(st)
    assert np.abs((hi1 - lo1) - (hi0 - lo0)).max() > 0
    assert st.status()[0] == 0
    sysd1 = systems.System(**{**sysd.__dict__, "lo": lo1, "L": hi1 - lo1})
    rel, rms = _water_forces_vs_oracle(oracle, st, sysd1, lo1, hi1 - lo1)
    assert rel < FORCE_RTOL, f"{rel:.3e} of RMS {rms:.3e}"


def test_mtk_npt_lj_follows_the_fp64_oracle():
    """FixNoseHoover.setPressure("ISO", P, tau): 30 NPT steps of an LJ fluid
    against the FP64 restatement of the reference's MTK propagator
    (oracle/mtk.py) from the same start: box, positions, barostat velocity
    and pressure"""
    from oracle.mtk import MTKLJ
    sysd = systems.lj_fcc(ncell=6, rho=0.8, jitter=0.05, seed=21, T=1.5)
    st, fx = systems.build_lj_state(sysd, rcut=2.5, skin=0.3, T=1.5, tau=0.5)
    nh = fx[1]
    nh.setPressure("ISO", 2.5, 0.5)
    ref = MTKLJ(sysd, T=1.5, tau=0.5, P=2.5, ptau=0.5)
    it = IntegratorVerlet(st)
    for chunk in range(3):
        it.run(10)
        if chunk:
            ref.restart()  # each run restarts the barostat at rest
        for _ in range(10):
            ref.step()
        ref.v *= ref.pending  # run end: the pending thermostat scale applied
        ref.pending = 1.0
        lo, hi = _box(st)
        np.testing.assert_allclose(hi - lo, ref.L, rtol=2e-6)
        assert nh.pressVel == pytest.approx(ref.pvel[0], rel=2e-3, abs=1e-6)
        assert nh.lastPressure == pytest.approx(ref.last_pressure, rel=2e-4)
        x, v, _ = st.getAtoms()
        d = _min_image(x - ref.x, ref.L)
        assert np.abs(d).max() < 5e-4, np.abs(d).max()
        assert np.abs(v - ref.v).max() < 5e-3 * np.abs(ref.v).max()
    assert st.status()[0] == 0


def test_mtk_npt_lj_reaches_the_set_pressure():
    """an LJ fluid started on a lattice at T = 1.5, rho = 0.7 (pressure -3.7)
    under the MTK barostat at P = 1: the box first shrinks, the mean pressure
    over the last stretch is the set point, and the density is the one the
    FP64 oracle's own 1,500-step run of the same propagator reaches on 864
    atoms (0.58)"""
    sysd = systems.lj_fcc(ncell=10, rho=0.7, jitter=0.05, seed=23, T=1.5)
    st, fx = systems.build_lj_state(sysd, rcut=2.5, skin=0.3, T=1.5, tau=0.5)
    nh = fx[1]
    nh.setPressure("ISO", 1.0, 0.5)
    lo0, hi0 = _box(st)
    it = IntegratorVerlet(st)
    it.run(100)
    lo1, hi1 = _box(st)
    assert np.prod(hi1 - lo1) < np.prod(hi0 - lo0)
    it.run(1400)
    ps, rho = [], []
    for _ in range(40):
        it.run(25)
        ps.append(nh.lastPressure)
        lo, hi = _box(st)
        rho.append(len(sysd.pos) / np.prod(hi - lo))
    assert abs(np.mean(ps) - 1.0) < 0.25, np.mean(ps)
    assert abs(np.mean(rho) - 0.58) < 0.03, np.mean(rho)
    assert st.status()[0] == 0
