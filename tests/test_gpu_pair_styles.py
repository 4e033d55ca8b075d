"""The other pair styles of compute_force_iso and the damped shifted force
charge term: FixLJCutFS (PairEvaluatorLJFS.h), FixLJCHARMM
(PairEvaluatorCHARMM.h), FixTICG (PairEvaluatorTICG.h), FixChargePairDSF
(ChargeEvaluatorDSF.h).  Per-site forces, energies and virials of the CUDA
path against the FP64 oracle (tables built by the oracle from the same set
parameters: mixing and defaults checked too) to FORCE_RTOL, and against the
reference's own compute_force_iso with the same evaluators, compiled from its
source, on the same list (both FP32: 2e-5 of the RMS force; 5e-4 with charges,
the reference's erfcf against this library's A&S erfc)."""
import numpy as np
import pytest

from md_engine_b200 import (Bounds, FixChargePairDSF, FixLJCHARMM, FixLJCut, FixLJCutFS, FixRigid, FixTICG, State,
                            Vector, systems)
from tests.helpers import FORCE_RTOL, force_err, water_bonds, water_small

pytestmark = pytest.mark.gpu


def _binary_lj(make_fix, setup, ncell=8, seed=5, rcut=2.5, skin=0.3):
    """a two-species LJ fluid (FCC lattice, jittered, species alternating)"""
    sysd = systems.lj_fcc(ncell=ncell, seed=seed, jitter=0.08)
    types = np.arange(len(sysd.pos)) % 2
    st = State()
    st.units.setLJ()
    st.bounds = Bounds(st, lo=Vector(*sysd.lo), hi=Vector(*(sysd.lo + sysd.L)))
    st.rCut = rcut
    st.padding = skin
    st.dt = 0.005
    st.atomParams.addSpecies(handle="A", mass=1.0, atomicNum=0)
    st.atomParams.addSpecies(handle="B", mass=2.0, atomicNum=0)
    st.addAtoms(["A" if t == 0 else "B" for t in types], sysd.pos, np.zeros(len(types)))
    fix = make_fix(st, "pair")
    setup(fix)
    st.activateFix(fix)
    return sysd, types, st


def _list_of(st):
    counts, nbr, tags = st.getNeighborList()
    return counts, nbr.astype(np.uint32) | (tags.astype(np.uint32) << 30)


def _check(oracle, st, sysd, types, table, kind, ck=0, q=None, qrc=0.0, alpha=0.0, dsf=None,
           coef=(1.0, 0.0, 0.0, 0.5), ref_tol=2e-5, real_units=False):
    st.prepare()
    st.computeForces(virialMode=1)
    x, _, fg = st.getAtoms()
    _, vg = st.virials()
    eg = st.potentialEnergy()[0]
    counts, ent = _list_of(st)
    qqr = oracle.REAL_UNITS["qqr_to_eng"] if real_units else 1.0
    ref = oracle.pair_forces_styles(x, types, q, table, sysd.L, counts, ent, coef=coef, lj_kind=kind, ck=ck,
                                    qrc=qrc, alpha=alpha, qqr_to_eng=qqr, dsf=dsf, want=("f", "virial", "energy"))
    rel, rms = force_err(fg, ref["f"])
    assert rms > 0.1
    assert rel < FORCE_RTOL, f"max force error {rel:.3e} of RMS {rms:.3e}"
    e_ref = float(ref["energy"].sum())
    # the per-site energies cancel in the sum (DSF charges): scale the FP32
    # tolerance by their magnitudes
    assert abs(eg - e_ref) < 1e-5 * float(np.abs(ref["energy"]).sum()) + 1e-4, (eg, e_ref)
    vr = ref["virial"].sum(0)
    assert np.abs(vg - vr).max() < 2e-4 * np.abs(vr).max()
    R = pytest.importorskip("oracle.refkernels")
    if R.available():
        xs4 = np.zeros((len(x), 4), np.float32)
        xs4[:, :3] = x
        xs4[:, 3] = np.asarray(types, np.int32).view(np.float32)
        dA, dshift = (float(dsf[0]), float(dsf[1])) if dsf is not None else (0.0, 0.0)
        fr = R.pair_styles(xs4, q, counts, ent, table.reshape(table.shape[0], -1), table.shape[1], sysd.lo,
                           sysd.L, coef[1:], kind if kind else 1, ck, qrc, alpha, qqr, dA, dshift)
        rms_r = np.sqrt(np.mean(np.sum(fr ** 2, 1)))
        assert np.max(np.linalg.norm(fg - fr, axis=1)) < ref_tol * rms_r


def _set_lj(fix, eps=(1.0, 0.6), sig=(1.0, 1.15), rcut=None):
    fix.setParameter("eps", "A", "A", eps[0])
    fix.setParameter("eps", "B", "B", eps[1])
    fix.setParameter("sig", "A", "A", sig[0])
    fix.setParameter("sig", "B", "B", sig[1])
    if rcut:
        fix.setParameter("rCut", "A", "B", rcut)


def test_lj_cut_fs_binary_mixture(oracle):
    sysd, types, st = _binary_lj(FixLJCutFS, lambda f: _set_lj(f, rcut=2.4))
    table = oracle.style_params(3, 2, eps={(0, 0): 1.0, (1, 1): 0.6}, sig={(0, 0): 1.0, (1, 1): 1.15}, rcut=2.5,
                                rcut_pairs={(0, 1): 2.4})
    _check(oracle, st, sysd, types, table, 3)


def test_lj_charmm_binary_mixture(oracle):
    def setup(f):
        _set_lj(f)
        f.setParameter("eps14", "A", "A", 0.3)
        f.setParameter("sig14", "B", "B", 0.9)
    sysd, types, st = _binary_lj(FixLJCHARMM, setup)
    table = oracle.style_params(4, 2, eps={(0, 0): 1.0, (1, 1): 0.6}, sig={(0, 0): 1.0, (1, 1): 1.15}, rcut=2.5,
                                eps14={(0, 0): 0.3}, sig14={(1, 1): 0.9}, coef14=0.5)
    _check(oracle, st, sysd, types, table, 4)


def test_ticg_binary_mixture(oracle):
    def setup(f):
        for a, b, c, r in (("A", "A", 2.0, 1.2), ("B", "B", 1.0, 1.3), ("A", "B", 3.0, 1.25)):
            f.setParameter("C", a, b, c)
            f.setParameter("rCut", a, b, r)
    sysd, types, st = _binary_lj(FixTICG, setup, rcut=1.3)
    table = oracle.style_params(5, 2, C={(0, 0): 2.0, (1, 1): 1.0, (0, 1): 3.0},
                                rcut_pairs={(0, 0): 1.2, (1, 1): 1.3, (0, 1): 1.25})
    _check(oracle, st, sysd, types, table, 5)


def _water_with(pair_fix_cls, setup, charge="dsf", coefs=(0.0, 0.0, 0.5), alpha=0.25, qrc=6.0):
    sysd = water_small(seed=19)
    st = State()
    st.units.setReal()
    st.bounds = Bounds(st, lo=Vector(*sysd.lo), hi=Vector(*(sysd.lo + sysd.L)))
    st.rCut = 6.5
    st.padding = 1.0
    st.dt = 2.0
    st.setSpecialNeighborCoefs(*coefs)
    for h, mm, z in sysd.species:
        st.atomParams.addSpecies(handle=h, mass=mm, atomicNum=z)
    st.addAtoms([sysd.species[t][0] for t in sysd.types], sysd.pos, sysd.q)
    pf = pair_fix_cls(st, "pair")
    setup(pf)
    st.activateFix(pf)
    dsf = FixChargePairDSF(st, "dsf")
    dsf.setParameters(alpha, qrc)
    st.activateFix(dsf)
    rigid = FixRigid(st, "rigid", "TIP4P/2005")
    for o, h1, h2, m in sysd.molecules:
        rigid.createRigid(o, h1, h2, m)
    st.activateFix(rigid)
    return sysd, st


def _water_lj(f, eps14=None):
    f.setParameter("sig", "OW", "OW", systems.SIG_OO)
    f.setParameter("eps", "OW", "OW", systems.EPS_OO)
    for a, b in (("HY", "HY"), ("OW", "HY"), ("OM", "OM")):
        f.setParameter("sig", a, b, 0.0)
        f.setParameter("eps", a, b, 0.0)
    if eps14 is not None:
        for a in ("OW", "HY", "OM"):
            f.setParameter("eps14", a, a, eps14)
            f.setParameter("sig14", a, a, 1.0)


def _water_table(oracle, kind, eps14=None):
    sig = {(0, 0): systems.SIG_OO, (1, 1): 0.0, (0, 1): 0.0, (2, 2): 0.0}
    eps = {(0, 0): systems.EPS_OO, (1, 1): 0.0, (0, 1): 0.0, (2, 2): 0.0}
    if kind == 4:
        e14 = {(a, a): eps14 for a in range(3)}
        s14 = {(a, a): 1.0 for a in range(3)}
        return oracle.style_params(4, 3, eps=eps, sig=sig, rcut=6.5, eps14=e14, sig14=s14)
    return oracle.style_params(kind, 3, eps=eps, sig=sig, rcut=6.5)


def test_dsf_charges_with_lj_cut_water(oracle):
    """LJ/cut + damped shifted force charges on rigid water (the excluded
    intramolecular pairs carry multiplier 0: no charge term, as the reference)"""
    sysd, st = _water_with(FixLJCut, _water_lj)
    assert int(st.pairForm) in (0, 1)
    st.prepare()
    assert int(st.pairForm) == 1  # DSF runs in the per-site form
    excl = oracle.exclusions_from_bonds(len(sysd.pos), water_bonds(sysd.molecules))
    assert excl is not None
    table = _water_table(oracle, 1)
    _check(oracle, st, sysd, sysd.types, table, 1, ck=2, q=sysd.q, qrc=6.0, alpha=0.25,
           dsf=oracle.dsf_constants(0.25, 6.0), ref_tol=5e-4, real_units=True)


def test_charmm_one_four_branch_with_dsf(oracle):
    """LJCHARMM takes its 1-4 parameters for pairs whose multiplier equals the
    1-4 coefficient (isNorm = multiplier != mult14): with 1-2 coefficient =
    1-4 coefficient = 0.5, water's bonded pairs use eps14/sig14"""
    sysd, st = _water_with(FixLJCHARMM, lambda f: _water_lj(f, eps14=0.05), coefs=(0.5, 0.0, 0.5))
    table = _water_table(oracle, 4, eps14=0.05)
    _check(oracle, st, sysd, sysd.types, table, 4, ck=2, q=sysd.q, qrc=6.0, alpha=0.25,
           dsf=oracle.dsf_constants(0.25, 6.0), coef=(1.0, 0.5, 0.0, 0.5), ref_tol=5e-4, real_units=True)


def test_lj_cut_fs_with_dsf_water(oracle):
    sysd, st = _water_with(FixLJCutFS, _water_lj)
    table = _water_table(oracle, 3)
    _check(oracle, st, sysd, sysd.types, table, 3, ck=2, q=sysd.q, qrc=6.0, alpha=0.25,
           dsf=oracle.dsf_constants(0.25, 6.0), ref_tol=5e-4, real_units=True)
