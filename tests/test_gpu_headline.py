"""Parity at the benchmarked configuration itself: rigid TIP4P/2005 (+E3B3),
4,096 molecules (16,384 sites), LJ + Ewald real space at 9 A with a 1 A skin,
P3M 64^3 order 5 -- the neighbour team, pair-kernel variant and FFT that the
timed step runs.  Forces, energies and the virial against the FP64 oracle;
the pair and E3B parts also against the reference's own kernels compiled
from its source, where they were built.  Two starts: the seeded lattice start
as generated, and the same system after 300 steps of dynamics (a disordered,
liquid-like configuration).  Tolerances as the 512-molecule tests."""
import numpy as np
import pytest

from md_engine_b200 import IntegratorVerlet, systems
from tests.helpers import FORCE_RTOL, force_err, oracle_water_params, water_bonds

pytestmark = pytest.mark.gpu

RCUT, SKIN, GRID = 9.0, 1.0, 64


def _state(e3b, steps, form=0):
    sysd = systems.water_tip4p2005(nside=16, seed=20261203)
    st, fx = systems.build_water_state(sysd, rcut=RCUT, skin=SKIN, grid=GRID, e3b=e3b, T=298.0, tau=25.0)
    st.pairForm = form
    st.prepare()
    if steps:
        IntegratorVerlet(st).run(steps)
    return sysd, st, fx


def _oracle_pair_p3m(O, sysd, x, alpha):
    excl = O.exclusions_from_bonds(len(x), water_bonds(sysd.molecules))
    xs4 = np.zeros((len(x), 4), np.float32)
    xs4[:, :3] = x
    O.wrap_f32(xs4, sysd.lo, sysd.L)
    cut = np.float32(float(np.float32(RCUT)) + SKIN)
    c, nb = O.nlist_cells(xs4, sysd.lo, sysd.L, cut, ids=np.arange(len(x)), excl=excl)
    pr = O.pair_forces(x, sysd.types, sysd.q, oracle_water_params(O, RCUT), sysd.L, c, nb, qrc=RCUT, alpha=alpha,
                       qqr_to_eng=O.REAL_UNITS["qqr_to_eng"], want=("f", "virial", "energy"))
    vir = pr["virial"].sum(0)
    frec, erec = O.p3m_forces(x, sysd.q, sysd.lo, sysd.L, (GRID,) * 3, alpha, want_energy=True, virial=vir)
    q2 = O.REAL_UNITS["qqr_to_eng"] * float(np.sum(sysd.q ** 2))
    return pr, frec, erec - alpha / np.sqrt(np.pi) * q2, vir


@pytest.mark.parametrize("steps,form", [(0, 0), (300, 0), (300, 1)])
def test_headline_forces_energy_virial_vs_fp64_oracle(oracle, steps, form):
    """form 0: the automatic choice (the molecule form for this all-rigid
    water, the benchmarked path); form 1: the per-site form (full-warp team)"""
    sysd, st, fx = _state(False, steps, form)
    assert int(st.pairForm) == (2 if form == 0 else 1)
    if form == 1:
        assert int(st.nThreadPerAtom) == 32
    st.computeForces(virialMode=1)
    x, _, fg = st.getAtoms()
    _, vg = st.virials()
    eg = st.potentialEnergy()
    alpha = fx["ewald"].alpha
    pr, frec, erec, vr = _oracle_pair_p3m(oracle, sysd, x, alpha)
    rel, rms = force_err(fg, pr["f"] + frec)
    assert rel < FORCE_RTOL, f"max force error {rel:.3e} of RMS {rms:.3e}"
    # the reciprocal part alone (own FFT) against the FP64 P3M
    rel_r, _ = force_err(fg - pr["f"], frec)
    assert rel_r < 5e-3, f"reciprocal force error {rel_r:.3e} of its RMS"
    e_pair = float(pr["energy"].sum())
    assert abs(eg[0] - e_pair) < 1e-4 * abs(e_pair)
    assert abs(eg[1] - erec) < 1e-4 * abs(erec)
    assert np.abs(vg - vr).max() < 2e-4 * np.abs(vr).max(), (vg, vr)


def test_headline_pair_kernel_matches_reference_kernel(oracle):
    R = pytest.importorskip("oracle.refkernels")
    if not R.available():
        pytest.skip("oracle/_ref/librefkernels.so not built")
    sysd, st, fx = _state(False, 300)
    st.computeForces()
    x, _, fg = st.getAtoms()
    counts, nbr, tags = st.getNeighborList()
    ent = nbr.astype(np.uint32) | (tags.astype(np.uint32) << 30)
    p = oracle_water_params(oracle, RCUT)
    pf = np.concatenate([p["rc2"].ravel(), p["eps24"].ravel(), p["sig6"].ravel()])
    xs4 = np.zeros((len(x), 4), np.float32)
    xs4[:, :3] = x
    xs4[:, 3] = np.asarray(sysd.types, np.int32).view(np.float32)
    alpha = fx["ewald"].alpha
    fr = R.pair_forces(xs4, sysd.q, counts, ent, pf, 3, sysd.lo, sysd.L, (0.0, 0.0, 0.5), 1, RCUT, alpha,
                       oracle.REAL_UNITS["qqr_to_eng"], ntpb=256, ntpa=32)
    frec = oracle.p3m_forces(x, sysd.q, sysd.lo, sysd.L, (GRID,) * 3, alpha)
    rms = np.sqrt(np.mean(np.sum(fr ** 2, 1)))
    err = np.max(np.linalg.norm(fg - (fr + frec), axis=1))
    assert err < 5e-4 * rms, err / rms


def test_headline_e3b_vs_fp64_oracle_and_reference_kernels(oracle):
    sysd, st, fx = _state(True, 300)
    st.computeForces()
    x, _, f_all = st.getAtoms()
    e = st.potentialEnergy()
    st.deactivateFix(fx["e3b"])
    st.prepare()
    st.putAtoms(positions=x)
    st.buildNeighborlists(force=True)
    st.computeForces()
    x2, _, f_no = st.getAtoms()
    d = x2 - x
    d -= sysd.L * np.rint(d / sysd.L)  # the rebuild may have wrapped atoms into the box
    assert np.abs(d).max() < 1e-5
    f_e3b = f_all - f_no
    fe, (e2, e3), npairs = oracle.e3b_forces(sysd.molecules, x, sysd.L, oracle.e3b_params("E3B3"))
    assert npairs > 10000
    rel, rms = force_err(f_e3b, fe)
    assert rel < 2e-3, f"E3B force error {rel:.3e} of RMS {rms:.3e}"
    assert abs(e[2] - e2) < 1e-4 * abs(e2) + 1e-6
    assert abs(e[3] - e3) < 1e-3 * abs(e3) + 1e-6
    R = pytest.importorskip("oracle.refkernels")
    if not R.available():
        return
    mol = sysd.molecules
    o = np.zeros((len(mol), 4), np.float32)
    o[:, :3] = x[mol[:, 0]]
    oracle.wrap_f32(o, sysd.lo, sysd.L)
    mc, mn = oracle.nlist_cells(o, sysd.lo, sysd.L, np.float32(6.2))
    xs4 = np.zeros((len(x), 4), np.float32)
    xs4[:, :3] = x
    xs4[:, 3] = np.asarray(sysd.types, np.int32).view(np.float32)
    fr = R.e3b_forces(xs4, mol, mc, mn, sysd.lo, sysd.L)
    rms_r = np.sqrt(np.mean(np.sum(fr ** 2, 1)))
    assert np.max(np.linalg.norm(f_e3b - fr, axis=1)) < 2e-3 * rms_r


@pytest.mark.parametrize("team", [1, 2, 4, 8, 16, 32])
def test_every_neighbour_team_matches_oracle(oracle, team):
    """nThreadPerAtom 1..32 (State tunable, the reference's NTPA sweep) on
    the 512-molecule water box: forces vs the FP64 oracle to FORCE_RTOL"""
    from tests.helpers import water_small
    sysd = water_small(seed=17)
    rc = 6.5
    st, fx = systems.build_water_state(sysd, rcut=rc, skin=1.0, grid=32, alpha=0.35, thermostat=False)
    st.pairForm = 1  # the per-site form: the team walks the per-site list
    st.nThreadPerAtom = team
    st.prepare()
    assert int(st.pairForm) == 1
    st.computeForces()
    x, _, fg = st.getAtoms()
    excl = oracle.exclusions_from_bonds(len(x), water_bonds(sysd.molecules))
    xs4 = np.zeros((len(x), 4), np.float32)
    xs4[:, :3] = x
    oracle.wrap_f32(xs4, sysd.lo, sysd.L)
    cut = np.float32(float(np.float32(rc)) + 1.0)
    c, nb = oracle.nlist_cells(xs4, sysd.lo, sysd.L, cut, ids=np.arange(len(x)), excl=excl)
    ref = oracle.pair_forces(x, sysd.types, sysd.q, oracle_water_params(oracle, rc), sysd.L, c, nb, qrc=rc,
                             alpha=0.35, qqr_to_eng=oracle.REAL_UNITS["qqr_to_eng"])["f"]
    ref = ref + oracle.p3m_forces(x, sysd.q, sysd.lo, sysd.L, (32, 32, 32), 0.35)
    rel, rms = force_err(fg, ref)
    assert rel < FORCE_RTOL, f"team {team}: max force error {rel:.3e} of RMS {rms:.3e}"


@pytest.mark.parametrize("e3b", [False, True])
def test_molecule_form_matches_per_site_form(oracle, e3b):
    """The molecule form (molecule-pair list, every site pair of a listed
    molecule pair, one warp per molecule) against the per-site form on the
    same positions: forces, energies and virials (both FP32)"""
    from tests.helpers import water_small
    sysd = water_small(seed=23)
    rc = 6.5
    res = {}
    x0 = None
    for form in (1, 2):
        st, fx = systems.build_water_state(sysd, rcut=rc, skin=1.0, grid=32, alpha=0.35, e3b=e3b,
                                           thermostat=False)
        st.pairForm = form
        st.prepare()
        if x0 is None:
            x0, _, _ = st.getAtoms()
        else:
            st.putAtoms(positions=x0)
            st.buildNeighborlists(force=True)
        assert int(st.pairForm) == form
        st.computeForces(virialMode=1)
        x, _, f = st.getAtoms()
        _, vir = st.virials()
        res[form] = (x, f, vir, st.potentialEnergy())
    (x1, f1, v1, e1), (x2, f2, v2, e2) = res[1], res[2]
    d = x2 - x1
    d -= sysd.L * np.rint(d / sysd.L)
    assert np.abs(d).max() < 1e-5
    rel, rms = force_err(f2, f1)
    assert rel < 2e-5, f"molecule vs per-site form: {rel:.3e} of RMS {rms:.3e}"
    assert np.abs(v2 - v1).max() < 2e-5 * np.abs(v1).max()
    assert np.allclose(e2, e1, rtol=1e-5, atol=1e-6)
