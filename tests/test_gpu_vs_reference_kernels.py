"""The B200 kernels against the REFERENCE's own kernels compiled from its
source for sm_100a (oracle/ref.mk: compute_force_iso, compute_E3B_force_*,
and GridGPU.cu's grid kernels from periodicWrap to assignNeighbors), run on
the same GPU with the same inputs.  Both are FP32, so the tolerance is tight
and the neighbour sets are compared bit for bit.  Skipped where oracle/_ref
was not built (reference sources absent)."""
import numpy as np
import pytest

from md_engine_b200 import systems
from tests.helpers import neighbor_cut, water_bonds, water_small

pytestmark = pytest.mark.gpu

R = pytest.importorskip("oracle.refkernels")
if not R.available():
    pytest.skip("oracle/_ref/librefkernels.so not built", allow_module_level=True)


def _params_flat(st_params):
    return np.concatenate([st_params["rc2"].ravel(), st_params["eps24"].ravel(), st_params["sig6"].ravel()])


def _xs4(x, types):
    xs4 = np.zeros((len(x), 4), np.float32)
    xs4[:, :3] = x
    xs4[:, 3] = np.asarray(types, np.int32).view(np.float32)
    return xs4


@pytest.mark.parametrize("case,ntpa", [("lj", 1), ("lj", 8), ("water", 1), ("water_mf", 4)])
def test_neighbor_list_matches_reference_gridgpu(oracle, case, ntpa):
    """this library's list against a forced build of the reference's own
    GridGPU kernels (GridGPU.cu:138-161 wrap, 190-293 bin and sort, 326-734
    count and assign) on the same positions: the same wrapped positions, the
    same per-atom counts and the same neighbour set of every atom (ids; the
    reference is built without exclusions, so the intramolecular pairs this
    library tags are compared as plain pairs)"""
    if case == "lj":
        sysd = systems.lj_fcc(ncell=12, seed=5, jitter=0.05)
        st, _ = systems.build_lj_state(sysd, rcut=2.5, skin=0.3)
        rcut, pad = 2.5, 0.3
    else:
        sysd = systems.water_tip4p2005(nside=12)
        st, _ = systems.build_water_state(sysd, rcut=9.0, skin=1.0, grid=32)
        st.pairForm = 2 if case == "water_mf" else 1
        rcut, pad = 9.0, 1.0
    st.prepare()
    x_pre, _, _ = st.getAtoms()
    st.buildNeighborlists(force=True)
    counts_g, nbr_g, _ = st.getNeighborList()
    cut = neighbor_cut(rcut, pad)
    rc, rn, rw = R.grid_build(np.asarray(x_pre, np.float32), sysd.lo, sysd.L, cut, ntpa=ntpa, maxn=1024)
    xs4 = np.zeros((len(x_pre), 4), np.float32)
    xs4[:, :3] = np.asarray(x_pre, np.float32)
    oracle.wrap_f32(xs4, sysd.lo, sysd.L)
    assert np.array_equal(rw, xs4[:, :3]), "periodicWrap differs from the oracle's wrap"
    assert np.array_equal(counts_g, rc), f"{int((counts_g != rc).sum())} atoms with other neighbour counts"
    mism = [i for i in range(len(rc))
            if not np.array_equal(np.sort(nbr_g[i, :rc[i]].astype(np.int64)), np.sort(rn[i, :rc[i]].astype(np.int64)))]
    assert not mism, f"{len(mism)} atoms with other neighbour sets (first {mism[:5]})"


def test_pair_kernel_matches_reference_kernel_lj(oracle):
    sysd = systems.lj_fcc(ncell=20, jitter=0.05)
    st, _ = systems.build_lj_state(sysd, rcut=2.5, skin=0.3)
    st.prepare()
    st.computeForces()
    x, _, fg = st.getAtoms()
    counts, nbr, tags = st.getNeighborList()
    ent = (nbr.astype(np.uint32) | (tags.astype(np.uint32) << 30))
    p = oracle.lj_params(1, {(0, 0): 1.0}, {(0, 0): 1.0}, 2.5)
    fr = R.pair_forces(_xs4(x, sysd.types), None, counts, ent, _params_flat(p), 1, sysd.lo, sysd.L,
                       (0.0, 0.0, 0.5), 1, 0.0, 0.0, 1.0)
    rms = np.sqrt(np.mean(np.sum(fr ** 2, 1)))
    assert np.max(np.linalg.norm(fg - fr, axis=1)) < 2e-5 * rms


def test_pair_kernel_matches_reference_kernel_water(oracle):
    sysd = water_small(seed=31)
    rcut = 6.5
    st, fx = systems.build_water_state(sysd, rcut=rcut, skin=1.0, grid=32, alpha=0.35, thermostat=False)
    st.deactivateFix(fx["ewald"])
    # pair + real-space Ewald only: re-enable the charge fix for the offload but
    # compare against reference pair kernel + our own P3M (identical input)
    st.activateFix(fx["ewald"])
    st.prepare()
    st.computeForces()
    x, _, fg = st.getAtoms()
    counts, nbr, tags = st.getNeighborList()
    ent = (nbr.astype(np.uint32) | (tags.astype(np.uint32) << 30))
    sig = {(0, 0): systems.SIG_OO, (1, 1): 0.0, (0, 1): 0.0, (2, 2): 0.0}
    eps = {(0, 0): systems.EPS_OO, (1, 1): 0.0, (0, 1): 0.0, (2, 2): 0.0}
    p = oracle.lj_params(3, sig, eps, rcut)
    fr = R.pair_forces(_xs4(x, sysd.types), sysd.q, counts, ent, _params_flat(p), 3, sysd.lo, sysd.L,
                       (0.0, 0.0, 0.5), 1, rcut, 0.35, oracle.REAL_UNITS["qqr_to_eng"])
    # add the reciprocal part from the FP64 oracle to both sides' comparison
    frec = oracle.p3m_forces(x, sysd.q, sysd.lo, sysd.L, (32, 32, 32), 0.35)
    rms = np.sqrt(np.mean(np.sum(fr ** 2, 1)))
    err = np.max(np.linalg.norm(fg - (fr + frec), axis=1))
    # real space: FP32 vs FP32 (reference uses __expf under --use_fast_math);
    # reciprocal: FP32 P3M vs FP64 oracle P3M
    assert err < 5e-4 * rms, err / rms


def test_e3b_kernels_match_reference_kernels(oracle):
    sysd = water_small(seed=33)
    st, fx = systems.build_water_state(sysd, rcut=6.5, skin=1.0, grid=32, e3b=True, alpha=0.35, thermostat=False)
    st.prepare()
    st.computeForces()
    x, _, f_all = st.getAtoms()
    st.deactivateFix(fx["e3b"])
    st.prepare()
    st.computeForces()
    _, _, f_no = st.getAtoms()
    f_e3b = f_all - f_no
    # the reference's molecule list: O-O pairs within rf + 1 A by its own
    # FP32 cell predicate on wrapped O positions (FixE3B.cu:349-406)
    mol = sysd.molecules
    o = np.zeros((len(mol), 4), np.float32)
    o[:, :3] = x[mol[:, 0]]
    oracle.wrap_f32(o, sysd.lo, sysd.L)
    mc, mn = oracle.nlist_cells(o, sysd.lo, sysd.L, np.float32(6.2))
    fr = R.e3b_forces(_xs4(x, sysd.types), mol, mc, mn, sysd.lo, sysd.L)
    rms = np.sqrt(np.mean(np.sum(fr ** 2, 1)))
    assert np.max(np.linalg.norm(f_e3b - fr, axis=1)) < 2e-3 * rms


def test_kernel_times_vs_reference_water4096(oracle):
    """Times the reference's own pair and E3B kernels (compiled from its
    source, the NTPB x NTPA sweep of Integrator::tune, Integrator.cu:275-276)
    against this library's on the same 4,096-molecule water inputs and prints
    both; the numbers are recorded in profiles/ (this is a measurement, the
    parity is checked by the tests above)."""
    sysd = systems.water_tip4p2005(nside=16)
    st, fx = systems.build_water_state(sysd, rcut=9.0, skin=1.0, grid=64, e3b=True, thermostat=False)
    st.pairBlocksPerSM = -1  # the pair kernel alone: the whole GPU (no room kept for the P3M chain)
    st.prepare()
    st.computeForces()
    x, _, _ = st.getAtoms()
    counts, nbr, tags = st.getNeighborList()
    ent = (nbr.astype(np.uint32) | (tags.astype(np.uint32) << 30))
    sig = {(0, 0): systems.SIG_OO, (1, 1): 0.0, (0, 1): 0.0, (2, 2): 0.0}
    eps = {(0, 0): systems.EPS_OO, (1, 1): 0.0, (0, 1): 0.0, (2, 2): 0.0}
    p = oracle.lj_params(3, sig, eps, 9.0)
    alpha = fx["ewald"].alpha
    xs4 = _xs4(x, sysd.types)
    best = None
    for ntpb in (64, 128, 256):
        for ntpa in (4, 8, 16, 32):
            _, ms = R.timed(R.pair_forces, 50, xs4, sysd.q, counts, ent, _params_flat(p), 3, sysd.lo, sysd.L,
                            (0.0, 0.0, 0.5), 1, 9.0, alpha, oracle.REAL_UNITS["qqr_to_eng"], ntpb=ntpb, ntpa=ntpa)
            if ms > 0 and (best is None or ms < best[0]):
                best = (ms, ntpb, ntpa)
    ours = st.timeStage("pair", iters=50, flushBytes=0)
    mol = sysd.molecules
    o = np.zeros((len(mol), 4), np.float32)
    o[:, :3] = x[mol[:, 0]]
    oracle.wrap_f32(o, sysd.lo, sysd.L)
    mc, mn = oracle.nlist_cells(o, sysd.lo, sysd.L, np.float32(6.2))
    best3 = None
    for ntpb in (64, 128, 256):
        for ntpa in (4, 8, 16, 32):
            _, ms = R.timed(R.e3b_forces, 50, xs4, mol, mc, mn, sysd.lo, sysd.L, ntpb=ntpb, ntpa=ntpa)
            if ms > 0 and (best3 is None or ms < best3[0]):
                best3 = (ms, ntpb, ntpa)
    ours3 = st.timeStage("e3b", iters=50, flushBytes=0)
    print(f"\npair: reference {best[0] * 1e3:.1f} us (NTPB {best[1]}, NTPA {best[2]}), this library {ours * 1e3:.1f} us")
    print(f"E3B: reference {best3[0] * 1e3:.1f} us (NTPB {best3[1]}, NTPA {best3[2]}), this library {ours3 * 1e3:.1f} us")
    assert best is not None and best3 is not None and ours > 0 and ours3 > 0


def _min_image(d, L):
    return d - L * np.rint(d / L)


def test_settle_matches_reference_kernels(oracle):
    """one velocity-Verlet step of rigid TIP4P/2005 water (thermostat off,
    molecule form): the positions after this library's first half against
    the reference's settlePositions + setMSite (FixRigid.cu:561-602,
    850-1132), and the velocities after its second half against the
    reference's settleVelocities (:658-848), each run on the same step's
    inputs (the kick and drift restated in FP32 as nve_v / nve_x,
    IntegratorVerlet.cu:23-61; the rigid-water constants from the
    reference's own FixRigid::populateRigidData)"""
    from md_engine_b200 import IntegratorVerlet
    sysd = water_small(seed=41)
    st, _ = systems.build_water_state(sysd, rcut=6.5, skin=1.0, grid=32, alpha=0.35, thermostat=False)
    st.prepare()
    assert int(st.pairForm) == 2
    x0, v0, f0 = st.getAtoms()
    IntegratorVerlet(st).run(1)
    x1, v2, f1 = st.getAtoms()
    mol = np.asarray(sysd.molecules)
    assert np.array_equal(mol.ravel(), np.arange(4 * len(mol))), "sites laid out O, H1, H2, M per molecule"
    # the step's second half folds M's force onto O and H (distributeMSite);
    # the first half after prepare kicks O and H with their own forces only,
    # as the reference's first step after prepareForRun does
    assert np.abs(f1[mol[:, 3]]).max() == 0, "M forces folded onto O, H"
    m = np.asarray(sysd.mass, np.float64)
    invm = np.where(m > 0, 1.0 / np.where(m > 0, m, 1.0), 0.0).astype(np.float32)
    masses = (m[mol[0, 0]], m[mol[0, 1]], m[mol[0, 3]])
    dt = float(st.dt)
    ftm = oracle.REAL_UNITS["ftm_to_v"]
    dtf = np.float32(0.5 * dt * np.float32(ftm))
    L = np.asarray(sysd.L)
    # first half: kick, drift, SETTLE, M
    vk = (np.asarray(v0, np.float32) + dtf * invm[:, None] * np.asarray(f0, np.float32)).astype(np.float32)
    xu = (np.asarray(x0, np.float32) + np.float32(dt) * vk).astype(np.float32)
    x1r, v1r = R.settle(x0, xu, vk, masses, sysd.lo, L, dt, ftm, 1)
    dx = np.abs(_min_image(np.asarray(x1) - x1r, L)).max()
    assert dx < 2e-5, f"positions after SETTLE differ by {dx:.2e} A"
    # second half: kick with the step's forces, SETTLE the velocities
    vk2 = (v1r.astype(np.float32) + dtf * invm[:, None] * np.asarray(f1, np.float32)).astype(np.float32)
    _, v2r = R.settle(x1r, x1r, vk2, masses, sysd.lo, L, dt, ftm, 2)
    sites = mol[:, :3].ravel()
    vrms = np.sqrt(np.mean(np.sum(v2r[sites] ** 2, 1)))
    dv = np.abs(np.asarray(v2)[sites] - v2r[sites]).max()
    assert dv < 1e-3 * vrms, f"velocities after SETTLE differ by {dv / vrms:.2e} of their RMS"
