"""Per-atom forces, energies and virials of the CUDA path vs the FP64 CPU
oracle (compute_force_iso PairEvaluateIso.h:8-207 with EvaluatorLJ,
EvaluatorWCA, ChargeEvaluatorEwald; P3M FixChargeEwald.cu; E3B
ThreeBodyE3B.h).  Tolerance: max per-atom error <= FORCE_RTOL * RMS force."""
import numpy as np
import pytest

from md_engine_b200 import systems
from tests.helpers import FORCE_RTOL, force_err, oracle_lj_params, oracle_water_params, water_bonds, water_small

pytestmark = pytest.mark.gpu


def _oracle_pair(O, st, sysd, params, rcut, padding, lj_kind=1, qrc=0.0, alpha=0.0, qqr=1.0, excl=None,
                 coef=(1.0, 0.0, 0.0, 0.5)):
    x, _, _ = st.getAtoms()
    xs4 = np.zeros((len(x), 4), np.float32)
    xs4[:, :3] = x
    cut = np.float32(float(np.float32(rcut)) + padding)
    counts, nbr = O.nlist_cells(xs4, sysd.lo, sysd.L, cut, ids=np.arange(len(x)), excl=excl)
    # the oracle works in FP64 on the same (float32-representable) positions
    return O.pair_forces(x, sysd.types, sysd.q, params, sysd.L, counts, nbr, coef=coef, lj_kind=lj_kind,
                         qrc=qrc, alpha=alpha, qqr_to_eng=qqr, want=("f", "virial", "energy")), x


@pytest.mark.parametrize("wca", [False, True])
def test_lj_wca_forces_32k(oracle, wca):
    sysd = systems.lj_fcc(ncell=20, jitter=0.05)
    st, _ = systems.build_lj_state(sysd, rcut=2.5, skin=0.3, wca=wca)
    st.prepare()
    st.computeForces(virialMode=1)
    x, _, fg = st.getAtoms()
    ref, _ = _oracle_pair(oracle, st, sysd, oracle_lj_params(oracle, sysd, 2.5, wca=wca), 2.5, 0.3,
                          lj_kind=2 if wca else 1)
    rel, rms = force_err(fg, ref["f"])
    assert rms > 1.0
    assert rel < FORCE_RTOL, f"max force error {rel:.3e} of RMS"
    vg, vsum = st.virials()
    vr = ref["virial"]
    assert np.allclose(vsum, vr.sum(0), rtol=1e-4, atol=1e-3 * np.abs(vr.sum(0)).max())
    e = st.potentialEnergy()
    assert abs(e[0] - ref["energy"].sum()) <= 1e-5 * abs(ref["energy"].sum()) + 1e-3


def _water_total(oracle, seed, alpha, rcut=6.5, pad=1.0, grid=32):
    sysd = water_small(seed=seed)
    st, fx = systems.build_water_state(sysd, rcut=rcut, skin=pad, grid=grid, alpha=alpha, thermostat=False)
    st.prepare()
    st.computeForces()
    x, _, fg = st.getAtoms()
    excl = oracle.exclusions_from_bonds(len(sysd.pos), water_bonds(sysd.molecules))
    ref, _ = _oracle_pair(oracle, st, sysd, oracle_water_params(oracle, rcut), rcut, pad, qrc=rcut, alpha=alpha,
                          qqr=oracle.REAL_UNITS["qqr_to_eng"], excl=excl)
    frec, erec = oracle.p3m_forces(x, sysd.q, sysd.lo, sysd.L, (grid,) * 3, alpha, want_energy=True)
    return st, sysd, x, fg, ref, frec, erec


def test_water_lj_ewald_real_plus_p3m_forces(oracle):
    """LJ + Ewald real space (with the excluded-pair correction) + P3M
    reciprocal: total per-atom force vs the FP64 oracle"""
    st, sysd, x, fg, ref, frec, _ = _water_total(oracle, 11, 0.35)
    rel, rms = force_err(fg, ref["f"] + frec)
    assert rel < FORCE_RTOL, f"max force error {rel:.3e} of RMS {rms:.3e}"


def test_p3m_reciprocal_force_and_energy(oracle):
    st, sysd, x, fg, ref, frec, erec = _water_total(oracle, 5, 0.4)
    rel, rms = force_err(fg - ref["f"], frec)
    assert rel < 5e-3, f"reciprocal force error {rel:.3e} of its RMS {rms:.3e}"
    e = st.potentialEnergy()
    Q2 = oracle.REAL_UNITS["qqr_to_eng"] * np.sum(sysd.q ** 2)
    erec_total = erec - 0.4 / np.sqrt(np.pi) * Q2
    assert abs(e[1] - erec_total) < 1e-4 * abs(erec_total)
    assert abs(e[0] - ref["energy"].sum()) < 1e-4 * abs(ref["energy"].sum())


def test_e3b_forces_vs_oracle(oracle):
    sysd = water_small(seed=7)
    rcut, pad = 6.5, 1.0
    st, fx = systems.build_water_state(sysd, rcut=rcut, skin=pad, grid=32, e3b=True, alpha=0.35, thermostat=False)
    st.prepare()
    st.computeForces()
    x, _, f_all = st.getAtoms()
    st.deactivateFix(fx["e3b"])
    st.prepare()
    st.computeForces()
    _, _, f_no = st.getAtoms()
    fe, (e2, e3), npairs = oracle.e3b_forces(sysd.molecules, x, sysd.L, oracle.e3b_params("E3B3"))
    assert npairs > 1000
    rel, rms = force_err(f_all - f_no, fe)
    assert rel < 2e-3, f"E3B force error {rel:.3e} of RMS {rms:.3e}"
    st.activateFix(fx["e3b"])
    st.prepare()
    e = st.potentialEnergy()
    assert abs(e[2] - e2) < 1e-4 * abs(e2) + 1e-6
    assert abs(e[3] - e3) < 1e-3 * abs(e3) + 1e-6


def test_water_e3b_total_virial_vs_oracle(oracle):
    """virialMode: the total virial of LJ + Ewald real space (pair kernel),
    the P3M reciprocal term (virials_cu, FixChargeEwald.cu:731-818) and E3B
    (two-body as the reference, plus the three-body term the reference leaves
    out) vs the FP64 oracle; the E3B part alone to 1e-3 of its size"""
    sysd = water_small(seed=9)
    rcut, pad, alpha, grid = 6.5, 1.0, 0.35, 32
    st, fx = systems.build_water_state(sysd, rcut=rcut, skin=pad, grid=grid, e3b=True, alpha=alpha,
                                       thermostat=False)
    st.prepare()
    st.computeForces(virialMode=1)
    _, v_all = st.virials()
    x, _, _ = st.getAtoms()
    excl = oracle.exclusions_from_bonds(len(sysd.pos), water_bonds(sysd.molecules))
    ref, _ = _oracle_pair(oracle, st, sysd, oracle_water_params(oracle, rcut), rcut, pad, qrc=rcut, alpha=alpha,
                          qqr=oracle.REAL_UNITS["qqr_to_eng"], excl=excl)
    v_pair = ref["virial"].sum(0)
    v_rec = np.zeros(6)
    oracle.p3m_forces(x, sysd.q, sysd.lo, sysd.L, (grid,) * 3, alpha, virial=v_rec)
    v_e3b = np.zeros(6)
    oracle.e3b_forces(sysd.molecules, x, sysd.L, oracle.e3b_params("E3B3"), virial=v_e3b)
    scale = max(np.abs(v_pair).max(), np.abs(v_rec).max(), np.abs(v_e3b).max())
    assert np.abs(v_all - (v_pair + v_rec + v_e3b)).max() < 2e-4 * scale, (v_all, v_pair, v_rec, v_e3b)
    st.deactivateFix(fx["e3b"])
    st.prepare()
    st.computeForces(virialMode=1)
    _, v_no = st.virials()
    assert np.abs(v_no - (v_pair + v_rec)).max() < 2e-4 * scale
    assert np.abs((v_all - v_no) - v_e3b).max() < 1e-3 * np.abs(v_e3b).max(), (v_all - v_no, v_e3b)


def test_pressure_vs_oracle_and_forces_kept(oracle):
    """mdx_pressure (DataComputerPressure.cu:76-92): (sum m v^2 + virial
    trace) / (3V) * nktv_to_press against the oracle's virials (pair, P3M,
    E3B), and the integrator's forces are the same before and after"""
    sysd = water_small(seed=12)
    rcut, pad, alpha, grid = 6.5, 1.0, 0.35, 32
    st, _ = systems.build_water_state(sysd, rcut=rcut, skin=pad, grid=grid, e3b=True, alpha=alpha,
                                      thermostat=False)
    st.prepare()
    _, _, f0 = st.getAtoms()
    p, v6 = st.pressure()
    x, v, f1 = st.getAtoms()
    assert np.array_equal(f0, f1)
    excl = oracle.exclusions_from_bonds(len(sysd.pos), water_bonds(sysd.molecules))
    ref, _ = _oracle_pair(oracle, st, sysd, oracle_water_params(oracle, rcut), rcut, pad, qrc=rcut, alpha=alpha,
                          qqr=oracle.REAL_UNITS["qqr_to_eng"], excl=excl)
    vir = ref["virial"].sum(0)
    oracle.p3m_forces(x, sysd.q, sysd.lo, sysd.L, (grid,) * 3, alpha, virial=vir)
    oracle.e3b_forces(sysd.molecules, x, sysd.L, oracle.e3b_params("E3B3"), virial=vir)
    mv2 = float(np.sum(sysd.mass[:, None] * np.asarray(v) ** 2))
    V = float(np.prod(sysd.L))
    p_ref = (mv2 * systems.MVV_TO_ENG_REAL + vir[:3].sum()) / (3.0 * V) * 68568.415
    scale = (mv2 * systems.MVV_TO_ENG_REAL + np.abs(vir[:3]).sum()) / (3.0 * V) * 68568.415
    assert abs(p - p_ref) < 5e-4 * scale, (p, p_ref)
