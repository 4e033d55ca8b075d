"""Neighbour list: the pair SET (with exclusion tags) must be bit-exact with
the reference's FP32 cell algorithm restated in oracle/oracle.c, on the same
wrapped positions (GridGPU.cu:138-161 wrap, 326-734 predicate)."""
import numpy as np
import pytest

from md_engine_b200 import systems
from tests.helpers import neighbor_cut, oracle_nlist_for, water_bonds

pytestmark = pytest.mark.gpu


def _compare(O, st, sysd, rcut, padding, excl=None):
    st.prepare()
    # prepare may move atoms after its first build (the initial SETTLE of
    # FixRigid); rebuild on the current positions and compare with those
    x_pre, _, _ = st.getAtoms()
    st.buildNeighborlists(force=True)
    x, _, _ = st.getAtoms()
    # the list is built on the wrapped float32 positions: the oracle's wrap of
    # the positions before and after the rebuild agree (the per-site form
    # wraps every atom in place; the molecule form keeps molecules whole and
    # wraps the per-site list's own sorted copy)
    xs4 = np.zeros((len(x_pre), 4), np.float32)
    xs4[:, :3] = np.asarray(x_pre, np.float32)
    O.wrap_f32(xs4, sysd.lo, sysd.L)
    xw = np.zeros((len(x), 4), np.float32)
    xw[:, :3] = np.asarray(x, np.float32)
    O.wrap_f32(xw, sysd.lo, sysd.L)
    assert np.array_equal(xs4[:, :3], xw[:, :3]), "periodic wrap differs"
    cut = neighbor_cut(rcut, padding)
    counts_o, nbr_o = oracle_nlist_for(O, xs4[:, :3], sysd.lo, sysd.L, cut,
                                       ids=np.arange(len(x)), excl=excl)
    counts_g, nbr_g, tags_g = st.getNeighborList()
    assert np.array_equal(counts_g, counts_o), "per-atom neighbour counts differ"
    mism = 0
    for i in range(len(x)):
        c = counts_o[i]
        oi = np.sort(nbr_o[i, :c] & O.EXCL_MASK).astype(np.int64)
        tag_o = {int(j & O.EXCL_MASK): int(j >> 30) for j in nbr_o[i, :c]}
        gi = nbr_g[i, :c].astype(np.int64)
        if not np.array_equal(gi, oi):
            mism += 1
            continue
        for k in range(c):
            assert tags_g[i, k] == tag_o[int(gi[k])], f"exclusion tag differs for pair {i},{gi[k]}"
    assert mism == 0, f"{mism} atoms with different neighbour sets"
    return counts_g


def test_lj_32k_pair_set_bit_exact(oracle):
    sysd = systems.lj_fcc(ncell=20)
    st, _ = systems.build_lj_state(sysd, rcut=2.5, skin=0.3)
    counts = _compare(oracle, st, sysd, 2.5, 0.3)
    assert 70 < counts.mean() < 85  # rho * 4/3 pi 2.8^3 = 77.6


def test_water_pair_set_and_exclusion_tags_bit_exact(oracle):
    sysd = systems.water_tip4p2005(nside=16)
    st, _ = systems.build_water_state(sysd, rcut=9.0, skin=1.0)
    excl = oracle.exclusions_from_bonds(len(sysd.pos), water_bonds(sysd.molecules))
    counts = _compare(oracle, st, sysd, 9.0, 1.0, excl=excl)
    assert counts.mean() > 500


def test_rebuild_after_motion_bit_exact(oracle):
    """positions moved by the integrator (and drifted out of the box) are
    wrapped and re-listed exactly as the reference would."""
    sysd = systems.lj_fcc(ncell=10, seed=5)
    st, _ = systems.build_lj_state(sysd, rcut=2.5, skin=0.3, interval=1)
    from md_engine_b200 import IntegratorVerlet
    IntegratorVerlet(st).run(25)
    st.buildNeighborlists(force=True)
    x, _, _ = st.getAtoms()
    xs4 = np.zeros((len(x), 4), np.float32)
    xs4[:, :3] = x.astype(np.float32)
    oracle.wrap_f32(xs4, sysd.lo, sysd.L)
    assert np.array_equal(xs4[:, :3].astype(np.float64), x)
    cut = neighbor_cut(2.5, 0.3)
    counts_o, nbr_o = oracle_nlist_for(oracle, xs4[:, :3], sysd.lo, sysd.L, cut)
    counts_g, nbr_g, _ = st.getNeighborList()
    assert np.array_equal(counts_g, counts_o)
    for i in range(len(x)):
        assert np.array_equal(nbr_g[i, :counts_g[i]], np.sort(nbr_o[i, :counts_o[i]]).astype(np.int32))


def test_small_box_edge_cases(oracle):
    """ragged sizes: 1 atom (no neighbours), 2 atoms across the boundary,
    a box with exactly 3 cells per side"""
    from md_engine_b200 import Bounds, FixLJCut, State, Vector
    for pos, L in ([[[1.0, 1.0, 1.0]], 9.0],
                   [[[0.1, 4.0, 4.0], [8.9, 4.0, 4.0]], 9.0],
                   [np.random.default_rng(3).uniform(0, 8.7, (300, 3)), 8.7]):
        pos = np.asarray(pos, np.float64)
        st = State()
        st.units.setLJ()
        st.bounds = Bounds(st, lo=Vector(0, 0, 0), hi=Vector(L, L, L))
        st.rCut = 2.5
        st.padding = 0.3
        st.atomParams.addSpecies("A", 1.0, 1)
        st.addAtoms(["A"] * len(pos), pos)
        lj = FixLJCut(st, "lj")
        lj.setParameter("sig", "A", "A", 1.0)
        lj.setParameter("eps", "A", "A", 1.0)
        st.activateFix(lj)
        st.prepare()
        x, _, _ = st.getAtoms()
        counts_o, nbr_o = oracle_nlist_for(oracle, x.astype(np.float32), np.zeros(3), np.full(3, L),
                                           neighbor_cut(2.5, 0.3))
        counts_g, nbr_g, _ = st.getNeighborList(maxPerAtom=max(int(counts_o.max()), 1))
        assert np.array_equal(counts_g, counts_o)
        for i in range(len(x)):
            assert np.array_equal(nbr_g[i, :counts_g[i]], np.sort(nbr_o[i, :counts_o[i]]).astype(np.int32))


def test_water_far_exclusions_bit_exact(oracle):
    """ids numbered site-major (all O, then all H1, H2, M): every exclusion
    partner lies thousands of ids away, outside the id window the build reads
    its exclusion depths from, so the tags come from the id list instead."""
    base = systems.water_tip4p2005(nside=8, seed=21)
    M = len(base.molecules)
    new_id = np.empty(4 * M, np.int64)
    for j, mol in enumerate(base.molecules):
        for k, old in enumerate(mol):
            new_id[old] = k * M + j
    order = np.argsort(new_id)
    sysd = systems.System(base.pos[order], base.vel[order], base.types[order], base.q[order],
                          base.mass[order], base.L, base.lo, base.species,
                          new_id[np.asarray(base.molecules)])
    st, _ = systems.build_water_state(sysd, rcut=6.5, skin=1.0, grid=32)
    excl = oracle.exclusions_from_bonds(len(sysd.pos), water_bonds(sysd.molecules))
    counts = _compare(oracle, st, sysd, 6.5, 1.0, excl=excl)
    assert counts.mean() > 150


@pytest.mark.parametrize("stencil,group", [(1, 2), (2, 4), (3, 2), (4, 4)])
def test_water_pair_set_every_stencil_and_home_group(oracle, stencil, group):
    """the list-build tunables (cells of >= cut/stencil, home atoms tested
    per warp) change the candidate walk, never the pair set or its tags"""
    sysd = systems.water_tip4p2005(nside=10)
    st, _ = systems.build_water_state(sysd, rcut=9.0, skin=1.0, grid=32)
    st.gridStencil = stencil
    st.gridHomeGroup = group
    excl = oracle.exclusions_from_bonds(len(sysd.pos), water_bonds(sysd.molecules))
    _compare(oracle, st, sysd, 9.0, 1.0, excl=excl)
    assert st.gridStencil == stencil and st.gridHomeGroup == group
