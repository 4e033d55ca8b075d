"""Pins of the CPU oracle against the reference's own known answers and
against analytic identities (CPU only).

Golden vectors from the reference's tests:
  * tests/Evaluators/test_PairEvaluatorLJ.py:72-152 -- LJ force at six
    separations (sigma 3, eps 6, rc 10), tolerance 1e-10 (FP64 build);
  * tests/Integrators/test_IntegratorVerlet.py:62-132 -- free-particle Verlet.
The reference's E3B, Ewald, WCA, SETTLE and neighbour-list tests are empty
stubs, so those parts are pinned by the identities below (and, on the GPU
box, by the reference's own kernels compiled from source, oracle/ref.mk).
"""
import ctypes
import math

import numpy as np
import pytest

from md_engine_b200 import systems


def _lj(O, sig, eps, rc, dr):
    out = np.zeros(3)
    dr = np.asarray(dr, np.float64)
    O.lib().orc_lj_force_single(sig, eps, rc, dr.ctypes.data_as(ctypes.c_void_p), out.ctypes.data_as(ctypes.c_void_p))
    return out


def test_lj_golden_vectors(oracle):
    sigma, epsilon, cutoff = 3.0, 6.0, 10.0
    A = np.array([10.0, 10.0, 10.0])
    Bs = [(9.0, 10.0, 10.0), (8.0, 10.0, 10.0), (7.0, 10.0, 10.0),
          (10.0 - (sigma * (2.0 ** (1.0 / 6.0))), 10.0, 10.0), (9.23472, 9.84752, 8.293478), (11.0, 9.0, 12.0)]
    sig6 = sigma ** 6
    sig12 = sig6 * sig6
    for B in Bs:
        dr = A - np.array(B)
        r = np.linalg.norm(dr)
        r2inv = 1.0 / r ** 2
        r6inv = r2inv ** 3
        expected = dr * r6inv * r2inv * 24.0 * epsilon * (2.0 * sig12 * r6inv - sig6)
        got = _lj(oracle, sigma, epsilon, cutoff, dr)
        diff = np.linalg.norm(got - expected)
        if diff > 1e-8:
            assert diff / np.linalg.norm(expected) <= 1e-10
        else:
            assert diff <= 1e-10


def test_lj_energy_shift_and_wca_zero_at_minimum(oracle):
    # LJ energy is zero at rc (shifted, PairEvaluatorLJ.h:38-58); WCA force is
    # zero at 2^(1/6) sigma and its energy there is 0 (PairEvaluatorWCA.h:13-38)
    for wca in (False, True):
        rc = 2.5
        p = oracle.lj_params(1, {(0, 0): 1.0}, {(0, 0): 1.0}, rc, wca=wca)
        rr = (2.0 ** (1.0 / 6.0)) if wca else rc - 1e-9
        x = np.array([[0.0, 0.0, 0.0], [rr, 0.0, 0.0]])
        c = np.array([1, 1], np.int32)
        nb = np.array([[1], [0]], np.uint32)
        out = oracle.pair_forces(x, np.zeros(2, int), None, p, np.full(3, 50.0), c, nb, lj_kind=2 if wca else 1,
                                 want=("f", "energy"))
        assert abs(out["energy"].sum()) < 1e-6
        if wca:
            assert np.abs(out["f"]).max() < 1e-9


def test_free_particle_verlet_fp64():
    # test_IntegratorVerlet.py:101-132 in FP64 (the oracle's precision)
    x, v, dt = 20.0, 1.0, 0.005
    for _ in range(10000):
        v += 0.5 * dt * 0.0
        x += dt * v
        v += 0.5 * dt * 0.0
    assert abs(x - (20.0 + dt * 10000 * 1.0)) <= 1e-10


def test_e3b_switching_continuity(oracle):
    prm = oracle.e3b_params("E3B3")

    def f(r):
        out = np.zeros(4)
        oracle.lib().orc_e3b_single(prm.ctypes.data_as(ctypes.c_void_p), float(r), out.ctypes.data_as(ctypes.c_void_p))
        return out

    rs, rf = prm[0], prm[1]
    for r0, expect in ((rs, 1.0), (rf, 0.0)):
        lo, hi = f(r0 - 1e-9), f(r0 + 1e-9)
        assert abs(lo[0] - hi[0]) < 1e-7 and abs(lo[0] - expect) < 1e-7
        assert abs(lo[1] - hi[1]) < 1e-6
    # threeBodyForce = -d/dr [s(r) exp(-k3 r)] (EvaluatorE3B.h:117-141)
    for r in (4.0, 5.05, 5.1, 5.19):
        h = 1e-6
        dE = (f(r + h)[2] - f(r - h)[2]) / (2 * h)
        assert abs(f(r)[3] / r * r + dE * 1.0) < 1e-6 * max(1.0, abs(dE))


def test_e3b_forces_are_energy_gradient(oracle):
    """E3B total energy (two-body + three-body, EvaluatorE3B.h:251-345) is
    consistent with the forces of ThreeBodyE3B.h (finite differences)."""
    sysd = systems.water_tip4p2005(nside=4, seed=3, density=1.2)
    x = sysd.pos.copy()
    prm = oracle.e3b_params("E3B3")
    f, (e2, e3), npairs = oracle.e3b_forces(sysd.molecules, x, sysd.L, prm)
    assert npairs > 10
    rng = np.random.default_rng(0)
    for atom in rng.choice(np.concatenate([sysd.molecules[:, 0], sysd.molecules[:, 1]]), 6, replace=False):
        for d in range(3):
            h = 1e-5
            xp = x.copy()
            xp[atom, d] += h
            xm = x.copy()
            xm[atom, d] -= h
            _, (a2, a3), _ = oracle.e3b_forces(sysd.molecules, xp, sysd.L, prm)
            _, (b2, b3), _ = oracle.e3b_forces(sysd.molecules, xm, sysd.L, prm)
            fd = -((a2 + a3) - (b2 + b3)) / (2 * h)
            assert abs(fd - f[atom, d]) < 1e-4 * max(1.0, abs(fd)), (atom, d, fd, f[atom, d])


def test_ewald_real_plus_p3m_vs_direct_ewald(oracle):
    """P3M reciprocal force (FixChargeEwald.cu order 5, optimal influence
    function) converges to the exact Ewald reciprocal sum"""
    rng = np.random.default_rng(4)
    n, L = 40, 12.0
    x = rng.uniform(0, L, (n, 3))
    q = rng.choice([-1.0, 1.0], n)
    q -= q.mean()
    alpha = 0.45
    f_p3m = oracle.p3m_forces(x, q, np.zeros(3), np.full(3, L), (32, 32, 32), alpha)
    f_ex, _ = oracle.ewald_recip_direct(x, q, np.full(3, L), alpha, kmax=10)
    rms = np.sqrt(np.mean(np.sum(f_ex ** 2, 1)))
    assert np.max(np.linalg.norm(f_p3m - f_ex, axis=1)) < 2e-3 * rms
    _, e_p3m = oracle.p3m_forces(x, q, np.zeros(3), np.full(3, L), (32, 32, 32), alpha, want_energy=True)
    _, e_ex = oracle.ewald_recip_direct(x, q, np.full(3, L), alpha, kmax=10)
    assert abs(e_p3m - e_ex) < 1e-3 * abs(e_ex)


def test_direct_ewald_force_is_gradient(oracle):
    rng = np.random.default_rng(5)
    x = rng.uniform(0, 8.0, (6, 3))
    q = np.array([1.0, -1.0, 0.5, -0.5, 1.0, -1.0])
    L = np.full(3, 8.0)
    f, _ = oracle.ewald_recip_direct(x, q, L, 0.5, kmax=6)
    h = 1e-5
    for i in range(3):
        xp = x.copy()
        xp[i, 0] += h
        xm = x.copy()
        xm[i, 0] -= h
        fd = -(oracle.ewald_recip_direct(xp, q, L, 0.5, 6)[1] - oracle.ewald_recip_direct(xm, q, L, 0.5, 6)[1]) / (2 * h)
        assert abs(fd - f[i, 0]) < 1e-5 * max(1.0, abs(fd))


def test_settle_restores_geometry_and_conserves_momentum(oracle):
    sysd = systems.water_tip4p2005(nside=4, seed=8)
    rd = oracle.RigidData("TIP4P/2005", systems.MASS_O, systems.MASS_H)
    mol = sysd.molecules
    x0 = sysd.pos[mol[:, :3]]
    rng = np.random.default_rng(2)
    v = rng.normal(0, 0.01, x0.shape)
    dt = 2.0
    x1 = x0 + v * dt + rng.normal(0, 0.002, x0.shape)
    xn, vn = oracle.settle_positions(x0, x1, v, sysd.L, rd, dt)
    for a, b, ref in ((0, 1, rd.r_OH), (0, 2, rd.r_OH), (1, 2, rd.r_HH)):
        d = np.linalg.norm(xn[:, a] - xn[:, b], axis=1)
        assert np.max(np.abs(d - ref)) < 1e-10
    m = np.array([rd.mO, rd.mH, rd.mH])
    com0 = np.einsum("k,mkd->md", m, x1)
    com1 = np.einsum("k,mkd->md", m, xn)
    assert np.max(np.abs(com0 - com1)) < 1e-10
    vs = oracle.settle_velocities(xn, vn, sysd.L, rd)
    p0 = np.einsum("k,mkd->md", m, vn)
    p1 = np.einsum("k,mkd->md", m, vs)
    assert np.max(np.abs(p0 - p1)) < 1e-12
    for a, b in ((0, 1), (0, 2), (1, 2)):
        rel = np.sum((vs[:, a] - vs[:, b]) * (xn[:, a] - xn[:, b]), 1)
        assert np.max(np.abs(rel)) < 1e-12


def test_nlist_cells_equals_brute_force(oracle):
    sysd = systems.lj_fcc(ncell=6, seed=1)
    rng = np.random.default_rng(0)
    xs4 = np.zeros((len(sysd.pos), 4), np.float32)
    xs4[:, :3] = sysd.pos + rng.normal(0, 0.2, sysd.pos.shape)
    oracle.wrap_f32(xs4, sysd.lo, sysd.L)
    cut = np.float32(2.8)
    c1, n1 = oracle.nlist_cells(xs4, sysd.lo, sysd.L, cut)
    c2, n2 = oracle.nlist_brute(xs4, sysd.L, cut)
    assert np.array_equal(c1, c2)
    for i in range(len(c1)):
        assert np.array_equal(np.sort(n1[i, :c1[i]]), np.sort(n2[i, :c2[i]]))


def test_exclusions_match_reference_bfs_semantics(oracle):
    """generateExclusionList (GridGPU.cu:1447-1518): TIP4P/2005 bonds O-H1,
    O-H2, H1-H2, O-M give every intra-molecular pair depth 1 or 2."""
    start, ent = oracle.exclusions_from_bonds(4, [(0, 1), (0, 2), (1, 2), (0, 3)])
    d = {}
    for i in range(4):
        for e in ent[start[i]:start[i + 1]]:
            d[(i, int(e & oracle.EXCL_MASK))] = int(e >> 30)
    assert d[(0, 1)] == 1 and d[(0, 2)] == 1 and d[(0, 3)] == 1 and d[(1, 2)] == 1
    assert d[(1, 3)] == 2 and d[(2, 3)] == 2 and d[(3, 1)] == 2
    assert len(d) == 12
    # a chain 0-1-2-3-4: depth 3 for 0-3, nothing for 0-4
    start, ent = oracle.exclusions_from_bonds(5, [(0, 1), (1, 2), (2, 3), (3, 4)])
    row = {int(e & oracle.EXCL_MASK): int(e >> 30) for e in ent[start[0]:start[1]]}
    assert row == {1: 1, 2: 2, 3: 3}


def test_p3m_alpha_secant_matches_library(oracle):
    """find_optimal_parameters (FixChargeEwald.cu:918-967) in the host C++ of
    the library equals the oracle's restatement (no GPU needed)."""
    from md_engine_b200 import FixChargeEwald
    sysd = systems.water_tip4p2005(nside=16)
    st, fx = systems.build_water_state(sysd, rcut=9.0, skin=1.0, grid=64, thermostat=False)
    a_lib = fx["ewald"].alpha
    a_orc = oracle.p3m_alpha(sysd.q, len(sysd.pos), sysd.L, (64, 64, 64), 9.0)
    assert abs(a_lib - a_orc) < 1e-9 * a_orc
    assert 0.2 < a_orc < 0.5


def test_nose_hoover_chain_conserved_quantity(oracle):
    """the chain integrator keeps its extended energy bounded for a harmonic
    bath (sanity of the restated FixNoseHoover.cu:795-866)"""
    nh = oracle.NoseHooverChain(1.0, 0.5, 300, 1.0, 0.005)
    nh.prepare(330.0)
    ke = 330.0
    for _ in range(2000):
        s = nh.integrate(True)
        ke *= s * s
        nh.ke = ke
        s = nh.integrate(False)
        ke *= s * s
    assert 150 < ke < 600


def test_oracle_per_pair_maths_vs_reference_functors(oracle):
    """the reference's own host-callable functors (EvaluatorLJ::force,
    EvaluatorE3B switching/threeBodyPairEnergy/threeBodyForce), compiled from
    its source by oracle/ref.mk, agree with the oracle to FP32 precision"""
    R = pytest.importorskip("oracle.refkernels")
    if not R.available():
        pytest.skip("oracle/_ref not built")
    rng = np.random.default_rng(7)
    for _ in range(50):
        dr = rng.uniform(-3, 3, 3)
        if np.linalg.norm(dr) < 2.0:
            continue
        r = R.lj_force_host(3.0, 6.0, 10.0, dr)
        o = _lj(oracle, 3.0, 6.0, 10.0, dr)
        assert np.max(np.abs(r - o)) <= 2e-6 * max(1.0, np.abs(o).max())
    prm = oracle.e3b_params("E3B3")
    for rr in np.linspace(0.8, 5.5, 60):
        a = R.e3b_single_host(rr)
        b = np.zeros(4)
        oracle.lib().orc_e3b_single(prm.ctypes.data_as(ctypes.c_void_p), float(rr), b.ctypes.data_as(ctypes.c_void_p))
        assert np.max(np.abs(a - b)) <= 2e-5 * max(1.0, np.abs(b).max())


def test_oracle_vs_committed_reference_functor_vectors(oracle):
    """golden vectors produced by the reference's own functors (compiled from
    its source; tests/golden/make_ref_functors.py) pin the oracle's per-pair
    LJ and E3B maths without the reference present"""
    import json
    import os
    with open(os.path.join(os.path.dirname(__file__), "golden", "ref_functors.json")) as f:
        g = json.load(f)
    assert len(g["lj"]) > 20 and len(g["e3b3_single"]) > 40
    for v in g["lj"]:
        o = _lj(oracle, v["sigma"], v["eps"], v["rcut"], np.array(v["dr"], np.float64))
        ref = np.array(v["force"])
        assert np.max(np.abs(ref - o)) <= 2e-6 * max(1.0, np.abs(o).max())
    prm = oracle.e3b_params("E3B3")
    for v in g["e3b3_single"]:
        b = np.zeros(4)
        oracle.lib().orc_e3b_single(prm.ctypes.data_as(ctypes.c_void_p), float(v["r"]), b.ctypes.data_as(ctypes.c_void_p))
        assert np.max(np.abs(np.array(v["out"]) - b)) <= 2e-5 * max(1.0, np.abs(b).max())


def test_e3b_and_p3m_virials_are_volume_derivatives(oracle):
    """every E3B force is a central pair force and the P3M reciprocal energy
    depends on positions and box through k and G(k): both virial traces equal
    -dE/d(eps) under the uniform scaling x -> (1 + eps) x, L -> (1 + eps) L"""
    sysd = systems.water_tip4p2005(nside=6, seed=3)
    x = sysd.pos.astype(np.float64)
    L = sysd.L.astype(np.float64)
    lo = sysd.lo.astype(np.float64)
    mol = np.asarray(sysd.molecules, np.int32)
    prm = oracle.e3b_params("E3B3")
    h = 1e-5

    vir = np.zeros(6)
    oracle.e3b_forces(mol, x, L, prm, virial=vir)

    def e3b(eps):
        _, (a, b), _ = oracle.e3b_forces(mol, x * (1 + eps), L * (1 + eps), prm)
        return a + b

    d = (e3b(h) - e3b(-h)) / (2 * h)
    assert abs(vir[:3].sum() + d) < 1e-6 * abs(d)

    sz, alpha = (32, 32, 32), 0.3
    vir = np.zeros(6)
    oracle.p3m_forces(x, sysd.q, lo, L, sz, alpha, virial=vir)

    def rec(eps):
        _, e = oracle.p3m_forces(lo + (x - lo) * (1 + eps), sysd.q, lo, L * (1 + eps), sz, alpha, want_energy=True)
        return e

    d = (rec(h) - rec(-h)) / (2 * h)
    assert abs(vir[:3].sum() + d) < 1e-6 * abs(d)


def _two_atom_style(oracle, kind, table, dr, coef=(1.0, 0.0, 0.0, 0.5), ck=0, q=None, qrc=0.0, alpha=0.0,
                    dsf=None):
    """force on atom 0 and the pair energy of a two-atom system (atom 1 at the
    origin, atom 0 at dr) by the oracle's pair styles; the per-atom energy
    of atom 0 is half of it (the reference half-counts each ordered pair)"""
    x = np.array([dr, [0.0, 0.0, 0.0]], np.float64)
    counts = np.array([1, 1], np.int32)
    nbr = np.array([[1], [0]], np.uint32)
    out = oracle.pair_forces_styles(x, [0, 0], q, table, [50.0, 50.0, 50.0], counts, nbr, coef=coef, lj_kind=kind,
                                    ck=ck, qrc=qrc, alpha=alpha, dsf=dsf, want=("f", "energy"))
    return out["f"][0], out["energy"].sum()


def test_ljfs_vs_committed_reference_functor_vectors(oracle):
    """the force-shifted LJ (FixLJCutFS) of the oracle against the reference's
    EvaluatorLJFS::force / energy on the parameters its forcePy forms, from
    the committed golden vectors; force and energy vanish at the cutoff"""
    import json
    import os
    with open(os.path.join(os.path.dirname(__file__), "golden", "ref_functors.json")) as f:
        g = json.load(f)
    assert len(g["ljfs"]) > 20
    for v in g["ljfs"]:
        tb = oracle.style_params(3, 1, eps={(0, 0): v["eps"]}, sig={(0, 0): v["sigma"]}, rcut=v["rcut"])
        dr = np.array(v["dr"], np.float64)
        fo, eo = _two_atom_style(oracle, 3, tb, dr)
        assert np.max(np.abs(np.array(v["force"]) - fo)) <= 2e-5 * max(1.0, np.abs(fo).max())
        # the functor adds F(rc) (rc - r) / 2 to the half-counted energy; the
        # oracle the force-consistent F(rc) (r - rc) / 2 its comment documents
        fcut, r = tb[3, 0, 0], np.linalg.norm(dr)
        assert abs(v["energy"] + fcut * (r - v["rcut"]) - 0.5 * eo) <= 2e-5 * max(1.0, abs(eo))
    tb = oracle.style_params(3, 1, eps={(0, 0): 0.8}, sig={(0, 0): 1.1}, rcut=2.5)
    f, e = _two_atom_style(oracle, 3, tb, np.array([2.5 - 1e-9, 0.0, 0.0]))
    assert abs(f[0]) < 1e-7 and abs(e) < 1e-9


def test_pair_style_forces_are_energy_gradients(oracle):
    """every pair style and charge term of the oracle: the force equals minus
    the gradient of its energy (central differences), away from the cutoff"""
    cases = [
        (1, oracle.style_params(1, 1, eps={(0, 0): 0.9}, sig={(0, 0): 1.0}, rcut=2.5), 0, 1.0),
        (3, oracle.style_params(3, 1, eps={(0, 0): 0.9}, sig={(0, 0): 1.0}, rcut=2.5), 0, 1.0),
        (4, oracle.style_params(4, 1, eps={(0, 0): 0.9}, sig={(0, 0): 1.0}, rcut=2.5,
                                eps14={(0, 0): 0.4}, sig14={(0, 0): 0.8}), 0, 1.0),
        (4, oracle.style_params(4, 1, eps={(0, 0): 0.9}, sig={(0, 0): 1.0}, rcut=2.5,
                                eps14={(0, 0): 0.4}, sig14={(0, 0): 0.8}), 0, 0.5),
        (5, oracle.style_params(5, 1, C={(0, 0): 3.0}, rcut_pairs={(0, 0): 2.0}), 0, 1.0),
        (0, np.zeros((3, 1, 1)), 2, 1.0),
    ]
    dsf = oracle.dsf_constants(0.25, 9.0)
    for kind, tb, ck, mult in cases:
        coef = (1.0, 0.5, 0.0, 0.5)
        q = np.array([0.7, -0.4])
        dr = np.array([1.05, 0.31, -0.22]) * (4.0 if ck else 1.0)
        tag_coef = (1.0, 0.0, 0.0, mult) if mult != 1.0 else coef
        f, _ = _two_atom_style(oracle, kind, tb, dr, coef=tag_coef if mult == 1.0 else (mult, 0.0, 0.0, mult),
                               ck=ck, q=q, qrc=9.0, alpha=0.25, dsf=dsf)
        h = 1e-6
        g = np.zeros(3)
        for d in range(3):
            e1 = np.array(dr)
            e2 = np.array(dr)
            e1[d] += h
            e2[d] -= h
            c = tag_coef if mult == 1.0 else (mult, 0.0, 0.0, mult)
            g[d] = -(_two_atom_style(oracle, kind, tb, e1, coef=c, ck=ck, q=q, qrc=9.0, alpha=0.25, dsf=dsf)[1] -
                     _two_atom_style(oracle, kind, tb, e2, coef=c, ck=ck, q=q, qrc=9.0, alpha=0.25, dsf=dsf)[1]) / (2 * h)
        # the pair energy is counted once per atom (half each): d/dx of the sum
        # is the force on atom 0
        assert np.allclose(f, g, rtol=1e-5, atol=1e-8), (kind, ck, mult, f, g)
