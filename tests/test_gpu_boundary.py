"""The reference-facing boundary pieces that the step does not exercise on
its own: the skin-displacement rebuild rule (setBuildFlag, GridGPU.cu:755-774),
the constraint validation (validateConstraints, FixRigid.cu:351-447), and the
raw kernel-level pair entry points -- mdx_pair_force_gridgpu on GridGPU's own
per-block padded list (EvaluatorWrapper.h:10-16, GridGPU.cu:777-821) against
the reference's compute_force_iso on the same list, and mdx_pair_force_raw
on this library's list against the stepped forces."""
import ctypes

import numpy as np
import pytest

from md_engine_b200 import MdxError, systems
from oracle import refkernels as R
from tests.helpers import FORCE_RTOL, force_err, oracle_water_params, water_small

pytestmark = pytest.mark.gpu


def test_skin_check_rebuilds_only_past_half_the_skin(oracle):
    sysd = systems.lj_fcc(ncell=6, seed=3, jitter=0.05)
    skin = 0.3
    st, _ = systems.build_lj_state(sysd, rcut=2.5, skin=skin)
    st.prepare()
    _, _, b0 = st.status()
    c0, n0, _ = st.getNeighborList()
    x0, _, _ = st.getAtoms()
    # just under skin/2 since the last build: no rebuild, same list
    x = x0.copy()
    x[7, 0] += 0.499 * skin
    st.putAtoms(positions=x)
    st.buildNeighborlists(force=False)
    _, _, b1 = st.status()
    c1, n1, _ = st.getNeighborList()
    assert b1 == b0
    assert np.array_equal(c0, c1) and np.array_equal(n0, n1)
    if R.available():
        # the reference's own setBuildFlag makes the same decision
        assert R.grid_skin_flag(x, x0, sysd.lo, sysd.L, skin) == 0
    # just over skin/2: rebuilt on the new positions, the oracle's pair set
    x[7, 0] = x0[7, 0] + 0.501 * skin
    if R.available():
        assert R.grid_skin_flag(x, x0, sysd.lo, sysd.L, skin) == 1
    st.putAtoms(positions=x)
    st.buildNeighborlists(force=False)
    _, _, b2 = st.status()
    assert b2 == b0 + 1
    xg, _, _ = st.getAtoms()
    xs4 = np.zeros((len(xg), 4), np.float32)
    xs4[:, :3] = xg
    cut = np.float32(float(np.float32(2.5)) + skin)
    co, _ = oracle.nlist_cells(xs4, sysd.lo, sysd.L, cut)
    c2, _, _ = st.getNeighborList()
    assert np.array_equal(c2, co)


def test_constraint_validation_flags_a_distorted_molecule():
    sysd = water_small(seed=5)
    st, fx = systems.build_water_state(sysd, rcut=6.5, skin=1.0, grid=32, alpha=0.35, thermostat=False)
    st.prepare()
    rigid = fx["rigid"]
    assert rigid.validateConstraints() == 0
    x, _, _ = st.getAtoms()
    bent = x.copy()
    h1 = int(sysd.molecules[10, 1])
    bent[h1] += np.array([0.02, 0.0, 0.0])  # an O-H bond 0.02 A off
    st.putAtoms(positions=bent)
    assert rigid.validateConstraints() == 1
    from md_engine_b200._lib import lib
    n = ctypes.c_uint32()
    assert lib().mdx_rigid_validate(st._h, rigid._h, ctypes.byref(n)) == 6  # MDX_ERR_NUMERIC
    st.putAtoms(positions=x)
    assert rigid.validateConstraints() == 0


def _gridgpu_layout(counts, nbr_ent, ntpb, ntpa):
    """GridGPU's list layout (GridGPU.cu:777-821): per block of ntpb threads,
    rows of ceil(max count / ntpa) * 32 entries per warp"""
    n = len(counts)
    per_block = ntpb // ntpa
    nblk = (n + per_block - 1) // per_block
    cum = np.zeros(nblk + 1, np.uint32)
    for b in range(nblk):
        mx = int(counts[b * per_block:(b + 1) * per_block].max())
        cum[b + 1] = cum[b] + ((mx + ntpa - 1) // ntpa) * 32
    wpb = ntpb // 32
    lst = np.zeros(int(cum[-1]) * wpb + 1, np.uint32)
    per_warp = 32 // ntpa
    for a in range(n):
        b, nth = divmod(a, per_block)
        mem = int(cum[b + 1] - cum[b])
        base = wpb * int(cum[b]) + mem * (nth // per_warp) + (nth % per_warp) * ntpa
        k = np.arange(counts[a])
        lst[base + k % ntpa + 32 * (k // ntpa)] = nbr_ent[a, :counts[a]]
    return cum, lst


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("ntpb,ntpa", [(256, 4), (128, 1), (64, 32)])
def test_pair_force_gridgpu_matches_reference_kernel_lj(oracle, ntpb, ntpa):
    torch = pytest.importorskip("torch")
    R = pytest.importorskip("oracle.refkernels")
    from md_engine_b200._lib import check, lib
    sysd = systems.lj_fcc(ncell=10, jitter=0.05, seed=4)
    st, _ = systems.build_lj_state(sysd, rcut=2.5, skin=0.3)
    st.prepare()
    x, _, _ = st.getAtoms()
    counts, nbr, tags = st.getNeighborList()
    ent = nbr.astype(np.uint32) | (tags.astype(np.uint32) << 30)
    cum, lst = _gridgpu_layout(counts, ent, ntpb, ntpa)
    n = len(x)
    xs4 = np.zeros((n, 4), np.float32)
    xs4[:, :3] = x
    p = oracle.lj_params(1, {(0, 0): 1.0}, {(0, 0): 1.0}, 2.5)
    pf = np.concatenate([p["rc2"].ravel(), p["eps24"].ravel(), p["sig6"].ravel()]).astype(np.float32)
    d_x, d_f = _dev(torch, xs4), torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    d_c, d_l, d_cum = _dev(torch, counts.astype(np.uint16)), _dev(torch, lst), _dev(torch, cum)
    d_p, d_v = _dev(torch, pf), torch.zeros((n, 6), dtype=torch.float32, device="cuda")
    lo = (ctypes.c_double * 3)(*sysd.lo)
    hi = (ctypes.c_double * 3)(*(sysd.lo + sysd.L))
    torch.cuda.synchronize()
    check(lib().mdx_pair_force_gridgpu(n, 1, d_x.data_ptr(), d_f.data_ptr(), d_c.data_ptr(), d_l.data_ptr(),
                                       d_cum.data_ptr(), 32, d_p.data_ptr(), 1, lo, hi, 0.0, 0.0, 0.5,
                                       d_v.data_ptr(), None, 0.0, 1, ntpb, ntpa, 1, 0.0, 1.0, None))
    torch.cuda.synchronize()
    fg = d_f.cpu().numpy()[:, :3].astype(np.float64)
    ref = oracle.pair_forces(x, sysd.types, None, p, sysd.L, counts, ent, want=("f", "virial"))
    rel, _ = force_err(fg, ref["f"])
    assert rel < FORCE_RTOL
    vg = d_v.cpu().numpy().astype(np.float64).sum(0)
    vr = ref["virial"].sum(0)
    assert np.abs(vg - vr).max() < 2e-4 * np.abs(vr).max()
    if R.available() and ntpa >= 2:  # the harness launches the reference's team kernels only
        fr = R.pair_forces(xs4, None, counts, ent, pf, 1, sysd.lo, sysd.L, (0.0, 0.0, 0.5), 1, 0.0, 0.0, 1.0,
                           ntpb=ntpb, ntpa=ntpa)
        rms = np.sqrt(np.mean(np.sum(fr ** 2, 1)))
        assert np.max(np.linalg.norm(fg - fr, axis=1)) < 2e-5 * rms


def test_pair_force_gridgpu_water_ewald(oracle):
    torch = pytest.importorskip("torch")
    from md_engine_b200._lib import check, lib
    sysd = water_small(seed=21)
    rc = 6.5
    st, fx = systems.build_water_state(sysd, rcut=rc, skin=1.0, grid=32, alpha=0.35, thermostat=False)
    st.prepare()
    x, _, _ = st.getAtoms()
    counts, nbr, tags = st.getNeighborList()
    ent = nbr.astype(np.uint32) | (tags.astype(np.uint32) << 30)
    cum, lst = _gridgpu_layout(counts, ent, 128, 8)
    n = len(x)
    xs4 = np.zeros((n, 4), np.float32)
    xs4[:, :3] = x
    xs4[:, 3] = np.asarray(sysd.types, np.int32).view(np.float32)
    p = oracle_water_params(oracle, rc)
    pf = np.concatenate([p["rc2"].ravel(), p["eps24"].ravel(), p["sig6"].ravel()]).astype(np.float32)
    d_x, d_f = _dev(torch, xs4), torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    d_c, d_l, d_cum = _dev(torch, counts.astype(np.uint16)), _dev(torch, lst), _dev(torch, cum)
    d_p, d_q = _dev(torch, pf), _dev(torch, np.asarray(sysd.q, np.float32))
    lo = (ctypes.c_double * 3)(*sysd.lo)
    hi = (ctypes.c_double * 3)(*(sysd.lo + sysd.L))
    qqr = oracle.REAL_UNITS["qqr_to_eng"]
    torch.cuda.synchronize()
    check(lib().mdx_pair_force_gridgpu(n, 1, d_x.data_ptr(), d_f.data_ptr(), d_c.data_ptr(), d_l.data_ptr(),
                                       d_cum.data_ptr(), 32, d_p.data_ptr(), 3, lo, hi, 0.0, 0.0, 0.5, None,
                                       d_q.data_ptr(), rc, 0, 128, 8, 1, 0.35, qqr, None))
    torch.cuda.synchronize()
    fg = d_f.cpu().numpy()[:, :3].astype(np.float64)
    ref = oracle.pair_forces(x, sysd.types, sysd.q, p, sysd.L, counts, ent, qrc=rc, alpha=0.35, qqr_to_eng=qqr)["f"]
    rel, _ = force_err(fg, ref)
    assert rel < FORCE_RTOL
    # a bad argument is an error, not a launch
    with pytest.raises(MdxError):
        check(lib().mdx_pair_force_gridgpu(n, 1, d_x.data_ptr(), d_f.data_ptr(), d_c.data_ptr(), d_l.data_ptr(),
                                           d_cum.data_ptr(), 16, d_p.data_ptr(), 3, lo, hi, 0.0, 0.0, 0.5, None,
                                           d_q.data_ptr(), rc, 0, 128, 8, 1, 0.35, qqr, None))


def test_pair_force_raw_on_own_layout_matches_oracle(oracle):
    torch = pytest.importorskip("torch")
    from md_engine_b200._lib import check, lib
    sysd = systems.lj_fcc(ncell=10, jitter=0.05, seed=6)
    st, _ = systems.build_lj_state(sysd, rcut=2.5, skin=0.3)
    st.prepare()
    x, _, _ = st.getAtoms()
    counts, nbr, tags = st.getNeighborList()
    ent = nbr.astype(np.uint32) | (tags.astype(np.uint32) << 30)
    team = 4
    G = 32 // team
    cap = int(((counts.max() + team - 1) // team) * team)
    n = len(x)
    groups = (n + G - 1) // G
    lst = np.zeros(groups * cap * G, np.uint32)
    for i in range(n):
        k = np.arange(counts[i])
        lst[(i // G) * cap * G + (k // team) * 32 + (i % G) * team + k % team] = ent[i, :counts[i]]
    xs4 = np.zeros((n, 4), np.float32)
    xs4[:, :3] = x
    p = oracle.lj_params(1, {(0, 0): 1.0}, {(0, 0): 1.0}, 2.5)
    pf = np.concatenate([p["rc2"].ravel(), p["eps24"].ravel(), p["sig6"].ravel()]).astype(np.float32)
    d_x, d_f = _dev(torch, xs4), torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    d_c, d_l, d_p = _dev(torch, counts.astype(np.uint32)), _dev(torch, lst), _dev(torch, pf)
    lo = (ctypes.c_double * 3)(*sysd.lo)
    hi = (ctypes.c_double * 3)(*(sysd.lo + sysd.L))
    coef = (ctypes.c_float * 3)(0.0, 0.0, 0.5)
    torch.cuda.synchronize()
    check(lib().mdx_pair_force_raw(n, d_x.data_ptr(), d_f.data_ptr(), None, d_c.data_ptr(), d_l.data_ptr(), team,
                                   cap, d_p.data_ptr(), 1, lo, hi, coef, 1, 0.0, 0.0, 1.0, None, 0, None))
    torch.cuda.synchronize()
    fg = d_f.cpu().numpy()[:, :3].astype(np.float64)
    ref = oracle.pair_forces(x, sysd.types, None, p, sysd.L, counts, ent)["f"]
    rel, _ = force_err(fg, ref)
    assert rel < FORCE_RTOL
