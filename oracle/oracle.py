"""CPU oracle for the DASH force hot path -- TEST INFRASTRUCTURE ONLY.

This module is the checker the CUDA path is compared against.  Only tests/,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import it;
the product package never does (it fails loudly instead of falling back here).

Contents (each function cites the reference code it restates):
  * ctypes bindings of oracle.c (FP32 neighbour predicate, FP64 pair / E3B forces)
  * exclusion lists by bond-graph depth          GridGPU.cu:1377-1518
  * P3M reciprocal space (FP64 numpy)            FixChargeEwald.cu:174-700, 918-967
  * direct Ewald reciprocal sum (pins the P3M)   standard Ewald formula
  * SETTLE positions / velocities, M-site        FixRigid.cu:475-1214, 1284-1436
  * velocity Verlet halves                       IntegratorVerlet.cu:23-61, 307-338, 610-627
  * Nose-Hoover chain (MTK, host FP64)           FixNoseHoover.cu:240-330, 413-604, 795-866, 1034-1056
  * a whole-step driver composing the above in the reference hook order
    (IntegratorVerlet.cu:694-754).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

EXCL_MASK = np.uint32(~(3 << 30) & 0xFFFFFFFF)

# unit constants, Units.cpp:5-32
REAL_UNITS = dict(boltz=0.0019872067, mvv_to_eng=48.88821291 * 48.88821291,
                  qqr_to_eng=332.06371, ftm_to_v=1.0 / (48.88821291 * 48.88821291))
LJ_UNITS = dict(boltz=1.0, mvv_to_eng=1.0, qqr_to_eng=1.0, ftm_to_v=1.0)


def build():
    """Compile oracle.c with its Makefile (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "_build", "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        P = ctypes.c_void_p
        I = ctypes.c_int
        D = ctypes.c_double
        F = ctypes.c_float
        L.orc_wrap_f32.argtypes = [I, P, P, P]
        L.orc_nlist_cells.argtypes = [I, P, P, P, F, P, P, P, P, P, I]
        L.orc_nlist_cells.restype = I
        L.orc_nlist_brute.argtypes = [I, P, P, F, P, P, I]
        L.orc_nlist_brute.restype = I
        L.orc_pair_forces.argtypes = [I, P, P, P, I, P, P, P, I, D, D, D, P, P, P, I, P, P, P, P]
        L.orc_pair_forces_styles.argtypes = [I, P, P, P, I, P, I, I, I, D, D, D, P, P, P, P, I, P, P, P, P]
        L.orc_e3b.argtypes = [I, P, P, P, P, P, P, P]
        L.orc_e3b.restype = I
        L.orc_lj_force_single.argtypes = [D, D, D, P, P]
        L.orc_e3b_single.argtypes = [P, D, P]
        L.orc_num_threads.restype = I
        L.orc_set_num_threads.argtypes = [I]
        _LIB = L
    return _LIB


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def set_threads(n):
    lib().orc_set_num_threads(int(n))


def num_threads():
    return lib().orc_num_threads()


# --------------------------------------------------------------------------
# neighbour list (FP32 predicate)
# --------------------------------------------------------------------------
def wrap_f32(xs4, lo, L):
    """GridGPU.cu:138-161 periodicWrap, in place on a float32 (n,4) array."""
    xs4 = np.ascontiguousarray(xs4, dtype=np.float32)
    lo = np.asarray(lo, np.float32)
    L = np.asarray(L, np.float32)
    lib().orc_wrap_f32(len(xs4), _p(xs4), _p(lo), _p(L))
    return xs4


def nlist_cells(xs4, lo, L, cut, ids=None, excl=None, maxn=None):
    """Neighbour list by the reference cell algorithm (GridGPU.cu:326-734).

    xs4: float32 (n,4), already wrapped.  Returns (counts int32[n],
    nbr uint32[n,maxn]) in input index order; entries carry the exclusion
    depth in bits 30-31 when ``excl`` = (start int32[maxId+2], ids uint32[]).
    """
    xs4 = np.ascontiguousarray(xs4, dtype=np.float32)
    n = len(xs4)
    lo = np.asarray(lo, np.float32)
    L = np.asarray(L, np.float32)
    if maxn is None:
        maxn = 64
    while True:
        counts = np.zeros(n, np.int32)
        nbr = np.zeros((n, maxn), np.uint32)
        ids_a = None if ids is None else np.ascontiguousarray(ids, np.int32)
        es = ei = None
        if excl is not None:
            es = np.ascontiguousarray(excl[0], np.int32)
            ei = np.ascontiguousarray(excl[1], np.uint32)
        mx = lib().orc_nlist_cells(n, _p(xs4), _p(lo), _p(L), np.float32(cut), _p(ids_a),
                                   _p(es), _p(ei), _p(counts), _p(nbr), maxn)
        if mx < 0:
            raise ValueError("box too small for the cell grid (needs >= 3 cells per side)")
        if mx <= maxn:
            return counts, nbr
        maxn = mx + 8


def nlist_brute(xs4, L, cut):
    xs4 = np.ascontiguousarray(xs4, dtype=np.float32)
    n = len(xs4)
    L = np.asarray(L, np.float32)
    maxn = 64
    while True:
        counts = np.zeros(n, np.int32)
        nbr = np.zeros((n, maxn), np.uint32)
        mx = lib().orc_nlist_brute(n, _p(xs4), _p(L), np.float32(cut), _p(counts), _p(nbr), maxn)
        if mx <= maxn:
            return counts, nbr
        maxn = mx + 8


def pair_sets(counts, nbr, ids):
    """Per-id sorted neighbour-id sets (the comparison GridGPU.cu:1109-1200 makes)."""
    ids = np.asarray(ids)
    out = {}
    for i in range(len(counts)):
        js = nbr[i, :counts[i]] & EXCL_MASK
        out[int(ids[i])] = np.sort(ids[js.astype(np.int64)])
    return out


# --------------------------------------------------------------------------
# exclusions (GridGPU.cu:1377-1518 generateExclusionList / handleExclusionsDistance)
# --------------------------------------------------------------------------
def exclusions_from_bonds(n_ids, bonds, max_depth=3):
    """Return (start int32[n_ids+1], entries uint32[]) with entry = id | depth<<30.

    Level 0 = bonded partners, level d = partners of level d-1 atoms that are
    not already closer (nor the atom itself); levels are listed in order and
    ids ascending within a level, as the reference's std::set iteration.
    """
    adj = [set() for _ in range(n_ids)]
    for a, b in bonds:
        adj[a].add(b)
        adj[b].add(a)
    levels = [[adj[i]] for i in range(n_ids)]
    for depth in range(1, max_depth):
        for i in range(n_ids):
            nxt = set()
            for k in levels[i][depth - 1]:
                nxt |= adj[k]
            closer = set([i])
            for d in range(depth):
                closer |= levels[i][d]
            levels[i].append(nxt - closer)
    start = np.zeros(n_ids + 1, np.int32)
    ent = []
    for i in range(n_ids):
        for d, s in enumerate(levels[i]):
            for j in sorted(s):
                ent.append(j | ((d + 1) << 30))
        start[i + 1] = len(ent)
    return start, np.asarray(ent, np.uint32)


# --------------------------------------------------------------------------
# pair forces (FP64)
# --------------------------------------------------------------------------
def pair_forces(x, types, q, params, L, counts, nbr, coef=(1.0, 0.0, 0.0, 0.5),
                lj_kind=1, qrc=0.0, alpha=0.0, qqr_to_eng=1.0, want=("f",)):
    """FP64 restatement of compute_force_iso / compute_energy_iso.

    params: dict with 'rc2','eps24','sig6' (ntypes x ntypes arrays).
    Returns dict with any of 'f' (n,3), 'virial' (n,6), 'energy' (n,).
    """
    x = np.ascontiguousarray(x, np.float64)
    n = len(x)
    nt = params["rc2"].shape[0]
    rc2 = np.ascontiguousarray(params["rc2"], np.float64)
    e24 = np.ascontiguousarray(params["eps24"], np.float64)
    s6 = np.ascontiguousarray(params["sig6"], np.float64)
    t = np.ascontiguousarray(types, np.int32)
    qq = np.ascontiguousarray(q if q is not None else np.zeros(n), np.float64)
    Ld = np.asarray(L, np.float64)
    c = np.ascontiguousarray(counts, np.int32)
    nb = np.ascontiguousarray(nbr, np.uint32)
    cf = np.asarray(coef, np.float64)
    f = np.zeros((n, 3)) if "f" in want else None
    v = np.zeros((n, 6)) if "virial" in want else None
    e = np.zeros(n) if "energy" in want else None
    lib().orc_pair_forces(n, _p(x), _p(t), _p(qq), nt, _p(rc2), _p(e24), _p(s6), int(lj_kind),
                          float(qrc), float(alpha), float(qqr_to_eng), _p(Ld), _p(c), _p(nb),
                          nb.shape[1], _p(cf), _p(f), _p(v), _p(e))
    out = {}
    if f is not None:
        out["f"] = f
    if v is not None:
        out["virial"] = v
    if e is not None:
        out["energy"] = e
    return out


def lj_params(ntypes, sig, eps, rcut, mixing="geometric", wca=False):
    """FixLJCut::prepareForRun / FixWCA::prepareForRun parameter processing
    (FixLJCut.cu:83-122, FixWCA.cu:60-106, FixPair.cpp:13-87).

    sig/eps: dict {(a,b): value} for explicitly set pairs; unset off-diagonal
    pairs are mixed (geometric eps; geometric or arithmetic sigma); rcut is the
    global cutoff (LJ) -- for WCA rc = sig*2^(1/6) per pair.
    """
    S = np.full((ntypes, ntypes), np.nan)
    E = np.full((ntypes, ntypes), np.nan)
    for (a, b), val in sig.items():
        S[a, b] = S[b, a] = val
    for (a, b), val in eps.items():
        E[a, b] = E[b, a] = val
    for a in range(ntypes):
        for b in range(ntypes):
            if np.isnan(E[a, b]):
                E[a, b] = math.sqrt(E[a, a] * E[b, b])
            if np.isnan(S[a, b]):
                S[a, b] = (S[a, a] + S[b, b]) / 2.0 if mixing == "arithmetic" else math.sqrt(S[a, a] * S[b, b])
    if wca:
        rc = S * 2.0 ** (1.0 / 6.0)
    else:
        rc = np.full((ntypes, ntypes), float(rcut))
    return dict(rc2=rc * rc, eps24=24.0 * E, sig6=S ** 6)


def style_params(kind, ntypes, eps=None, sig=None, rcut=None, rcut_pairs=None, eps14=None, sig14=None, C=None,
                 mixing="geometric", coef14=0.5):
    """The processed parameter tables (np x ntypes x ntypes, FP64, the
    reference's paramOrder) of a pair style: 1 LJ/cut, 3 force-shifted LJ,
    4 CHARMM, 5 TICG -- prepareForRun of FixLJCut.cu:83-122,
    FixLJCutFS.cu:84-130 (F(rc) as EvaluatorLJFS::forcePy forms it,
    PairEvaluatorLJFS.cu), FixLJCHARMM.cu:113-180 (unset 1-4 diagonal
    entries are the ordinary ones times the 1-4 coefficient), FixTICG.cu:68-83
    (no mixing).  Dicts {(a, b): value} for the explicitly set pairs; rcut is
    state.rCut, rcut_pairs the per-pair rCut overrides."""
    def table(d, mix, diag_default=None):
        T = np.full((ntypes, ntypes), np.nan)
        for (a, b), val in (d or {}).items():
            T[a, b] = T[b, a] = val
        if diag_default is not None:
            for a in range(ntypes):
                if np.isnan(T[a, a]):
                    T[a, a] = diag_default(a)
        for a in range(ntypes):
            for b in range(ntypes):
                if np.isnan(T[a, b]):
                    if mix == "max":
                        T[a, b] = max(T[a, a], T[b, b])
                    elif mix == "arithmetic":
                        T[a, b] = (T[a, a] + T[b, b]) / 2.0
                    else:
                        T[a, b] = math.sqrt(T[a, a] * T[b, b])
        return T
    if kind == 5:
        Ct = table(C, None)
        R = table(rcut_pairs, None)
        return np.stack([R * R, Ct])
    E = table(eps, "geometric")
    S = table(sig, "arithmetic" if mixing == "arithmetic" else "geometric")
    R = table(rcut_pairs, "max", lambda a: float(rcut))
    rc2, e24, s6 = R * R, 24.0 * E, S ** 6
    out = [rc2, e24, s6]
    if kind == 3:
        p1, p2 = e24 * 2.0 * s6 * s6, e24 * s6
        r2inv = 1.0 / rc2
        out.append(r2inv ** 3 * np.sqrt(r2inv) * (p1 * r2inv ** 3 - p2))
    if kind == 4:
        E0 = {(a, a): E[a, a] * coef14 for a in range(ntypes)}
        S0 = {(a, a): S[a, a] * coef14 for a in range(ntypes)}
        E0.update(eps14 or {})
        S0.update(sig14 or {})
        E14 = table(E0, "geometric")
        S14 = table(S0, "arithmetic" if mixing == "arithmetic" else "geometric")
        out += [24.0 * E14, S14 ** 6]
    return np.stack(out)


def dsf_constants(alpha, rc):
    """FixChargePairDSF::setParameters: (2 alpha/sqrt(pi), shift,
    erfc(alpha rc)/rc, rc), shift = erfc(alpha rc)/rc^2 + A exp(-alpha^2 rc^2)/rc"""
    A = 2.0 / math.sqrt(math.pi) * alpha
    shift = math.erfc(alpha * rc) / (rc * rc) + A * math.exp(-alpha * alpha * rc * rc) / rc
    return np.array([A, shift, math.erfc(alpha * rc) / rc, rc], np.float64)


def pair_forces_styles(x, types, q, table, L, counts, nbr, coef=(1.0, 0.0, 0.0, 0.5), lj_kind=1, ck=0, qrc=0.0,
                       alpha=0.0, qqr_to_eng=1.0, dsf=None, want=("f",)):
    """FP64 compute_force_iso with any of the pair styles (table from
    style_params; lj_kind 0 none, 1, 3, 4, 5) and charge evaluators (ck 0
    none, 1 Ewald, 2 DSF with dsf from dsf_constants)."""
    x = np.ascontiguousarray(x, np.float64)
    n = len(x)
    tb = np.ascontiguousarray(table, np.float64)
    npar, nt = tb.shape[0], tb.shape[1]
    t = np.ascontiguousarray(types, np.int32)
    qq = np.ascontiguousarray(q if q is not None else np.zeros(n), np.float64)
    Ld = np.asarray(L, np.float64)
    c = np.ascontiguousarray(counts, np.int32)
    nb = np.ascontiguousarray(nbr, np.uint32)
    cf = np.asarray(coef, np.float64)
    ds = np.ascontiguousarray(dsf if dsf is not None else np.zeros(4), np.float64)
    f = np.zeros((n, 3)) if "f" in want else None
    v = np.zeros((n, 6)) if "virial" in want else None
    e = np.zeros(n) if "energy" in want else None
    lib().orc_pair_forces_styles(n, _p(x), _p(t), _p(qq), nt, _p(tb), npar, int(lj_kind), int(ck), float(qrc),
                                 float(alpha), float(qqr_to_eng), _p(ds), _p(Ld), _p(c), _p(nb), nb.shape[1], _p(cf),
                                 _p(f), _p(v), _p(e))
    out = {}
    if f is not None:
        out["f"] = f
    if v is not None:
        out["virial"] = v
    if e is not None:
        out["energy"] = e
    return out


# --------------------------------------------------------------------------
# E3B (FP64)
# --------------------------------------------------------------------------
KJ_TO_KCAL = 0.23900573614


def e3b_params(style="E3B3"):
    """FixE3B::createEvaluator (FixE3B.cu:515-593) in kcal/mol and Angstrom,
    plus the molecule-list radius rf + padding (FixE3B.cu:29, 657) and
    RMAX_E3B (ThreeBodyE3B.h:16)."""
    if style == "E3B3":
        E2, Ea, Eb, Ec = 453000.0, 150.0, -1005.0, 1880.0
    elif style == "E3B2":
        E2, Ea, Eb, Ec = 2349000.0, 1745.7, -4565.0, 7606.8
    else:
        raise ValueError(style)
    k = KJ_TO_KCAL
    return np.array([5.0, 5.2, E2 * k, Ea * k, Eb * k, Ec * k, 4.872, 1.907, 6.2, 6.1572], np.float64)


def e3b_forces(mol, x, L, prm, natoms=None, virial=None):
    """Returns (f (natoms,3), (E2body, E3body), n_threebody_pairs).  virial: a
    6-vector (xx yy zz xy xz yz) the total E3B virial is added to -- two-body
    as the reference, plus the three-body pair forces."""
    x = np.ascontiguousarray(x, np.float64)
    natoms = len(x) if natoms is None else natoms
    m = np.ascontiguousarray(mol, np.int32)
    f = np.zeros((natoms, 3))
    e = np.zeros(2)
    Ld = np.asarray(L, np.float64)
    pr = np.ascontiguousarray(prm, np.float64)
    vir = np.zeros(6)
    npairs = lib().orc_e3b(len(m), _p(m), _p(x), _p(Ld), _p(pr), _p(f), _p(e), _p(vir))
    if virial is not None:
        virial += vir
    return f, (e[0], e[1]), npairs


# --------------------------------------------------------------------------
# P3M (FixChargeEwald.cu), FP64 numpy restatement
# --------------------------------------------------------------------------
_AMP = [
    [2.0 / 3.0, 0, 0, 0, 0, 0, 0],
    [1.0 / 50.0, 5.0 / 294.0, 0, 0, 0, 0, 0],
    [1.0 / 588.0, 7.0 / 1440.0, 21.0 / 3872.0, 0, 0, 0, 0],
    [1.0 / 4320.0, 3.0 / 1936.0, 7601.0 / 2271360.0, 143.0 / 28800.0, 0, 0, 0],
    [1.0 / 23232.0, 7601.0 / 12628160.0, 143.0 / 69120.0, 517231.0 / 106536960.0,
     106640677.0 / 11737571328.0, 0, 0],
]


def p3m_alpha(q, natoms, L, sz, rcut, order=5, qqr_to_eng=REAL_UNITS["qqr_to_eng"], ref_float=False, q2=None):
    """FixChargeEwald::find_optimal_parameters (FixChargeEwald.cu:918-967):
    secant solve of DeltaF_k(alpha) = DeltaF_real(alpha) (:865-883), in FP64
    (the library's precision).  ref_float: in the reference's own precision
    -- its box sides, mesh spacings, cutoff, total squared charge and alpha
    are floats (real3 L, h; real r_cut, total_Q2, alpha; FixChargeEwald.h),
    so L.x * L.x and the product under DeltaF_real's square root are float
    arithmetic.  q2: the total squared charge times qqr_to_eng, in place of
    the charges q."""
    Q2 = qqr_to_eng * float(np.sum(np.asarray(q, np.float64) ** 2)) if q2 is None else float(q2)
    amp = _AMP[order - 1]
    if ref_float:
        f32 = np.float32
        Lf = np.asarray(L, np.float32)
        hf = Lf / np.asarray(sz, np.float32)
        rcf, Q2f = f32(rcut), f32(Q2)
        L, h, rcut, Q2 = Lf.astype(np.float64), hf.astype(np.float64), float(rcf), float(Q2f)
        invL2 = 1.0 / (Lf * Lf).astype(np.float64)
        vol = f32(f32(f32(f32(natoms) * rcf) * Lf[0]) * Lf[1]) * Lf[2]
        pre_r = float(f32(f32(2) * Q2f) / np.sqrt(f32(vol)))
    else:
        L = np.asarray(L, np.float64)
        h = L / np.asarray(sz, np.float64)
        invL2 = 1.0 / (L * L)
        pre_r = 2 * Q2 / math.sqrt(natoms * rcut * L[0] * L[1] * L[2])

    def dk(a):
        s = np.zeros(3)
        for m in range(order):
            s += amp[m] * (h * a) ** (2 * m)
        return Q2 / 3.0 * float(np.sum(invL2 * (a * h) ** order *
                                       np.sqrt(a * L / natoms * math.sqrt(2.0 * math.pi) * s)))

    def dr(a):
        return pre_r * math.exp(-a * a * rcut * rcut)

    xa, xb = 0.0, 4.79853 / rcut
    ya, yb = dk(xa) - dr(xa), dk(xb) - dr(xb)
    it = 0
    while abs(yb) / dr(xb) > 1e-5 and it < 100:
        kinv = (xb - xa) / (yb - ya)
        ya, xa = yb, xb
        xb = xa - ya * kinv
        yb = dk(xb) - dr(xb)
        it += 1
    return float(np.float32(xb)) if ref_float else xb


def _W5(i, x):
    x2 = x * x
    x4 = x2 * x2
    if i == -2:
        return (1.0 / 384.0) * (1.0 - 8.0 * x + 24.0 * x2 - 32.0 * x * x2 + 16.0 * x4)
    if i == -1:
        return (1.0 / 96.0) * (19.0 - 44.0 * x + 24.0 * x2 + 16.0 * x * x2 - 16.0 * x4)
    if i == 0:
        return (1.0 / 192.0) * (115.0 - 120.0 * x2 + 48.0 * x4)
    if i == 1:
        return (1.0 / 96.0) * (19.0 + 44.0 * x + 24.0 * x2 - 16.0 * x * x2 - 16.0 * x4)
    return (1.0 / 384.0) * (1.0 + 8.0 * x + 24.0 * x2 + 32.0 * x * x2 + 16.0 * x4)


def _kvec(L, sz):
    ks = []
    for d in range(3):
        idx = np.arange(sz[d])
        k = 2.0 * math.pi * idx / L[d]
        k = np.where(idx > sz[d] // 2, 2.0 * math.pi * (idx - sz[d]) / L[d], k)
        ks.append(k)
    return ks


def p3m_green(L, sz, alpha, order=5):
    """Green_function_cu (FixChargeEwald.cu:314-366) with sum_limits from
    calc_Green_function (FixChargeEwald.cu:1124)."""
    L = np.asarray(L, np.float64)
    h = L / np.asarray(sz)
    lim = int(alpha * (h[0] * h[1] * h[2]) ** (1.0 / 3.0) / 3.14159 * math.sqrt(-math.log(10e-7))) + 1
    kx, ky, kz = np.meshgrid(*_kvec(L, sz), indexing="ij")
    k2 = kx * kx + ky * ky + kz * kz
    s1 = np.zeros(k2.shape)
    s2 = np.zeros(k2.shape)
    f4a = 0.25 / alpha / alpha

    def sinc(v):
        return np.where(np.abs(v) < 0.1, 1.0 - v * v / 6.0 + v ** 4 / 120.0 - v ** 6 / 5040.0,
                        np.sin(v) / np.where(v == 0, 1.0, v))

    for ix in range(-lim, lim + 1):
        for iy in range(-lim, lim + 1):
            for iz in range(-lim, lim + 1):
                mx = kx + 2 * math.pi * ix / h[0]
                my = ky + 2 * math.pi * iy / h[1]
                mz = kz + 2 * math.pi * iz / h[2]
                mm = mx * mx + my * my + mz * mz
                W = sinc(mx * h[0] * 0.5) * sinc(my * h[1] * 0.5) * sinc(mz * h[2] * 0.5)
                W2 = W ** (2 * order)
                with np.errstate(divide="ignore", invalid="ignore"):
                    s1 += np.where(mm > 0, 4.0 * math.pi * np.exp(-mm * f4a) *
                                   (kx * mx + ky * my + kz * mz) / np.where(mm > 0, mm, 1.0) * W2, 0.0)
                s2 += W2
    with np.errstate(divide="ignore", invalid="ignore"):
        G = np.where(k2 != 0, s1 / (s2 * s2) / np.where(k2 != 0, k2, 1.0), 0.0)
    return G


def _p3m_stencil(x, lo, L, sz):
    """nearest grid point and fractional offsets (FixChargeEwald.cu:181-190)."""
    x = np.asarray(x, np.float64) - np.asarray(lo, np.float64)
    h = np.asarray(L, np.float64) / np.asarray(sz)
    ng = np.floor((x + 0.5 * h) / h).astype(np.int64)  # make_int3 truncates; x+h/2 > 0 here
    d = x / h - ng
    return ng, d


def p3m_forces(x, q, lo, L, sz, alpha, order=5, qqr_to_eng=REAL_UNITS["qqr_to_eng"],
               G=None, want_energy=False, virial=None):
    """Reciprocal-space P3M force (FixChargeEwald::compute, order 5), FP64.

    Spread (map_charge_to_grid_order_5_cu) -> FFT -> ik G rho (E_field_cu) ->
    3 inverse FFTs -> gather (Ewald_long_range_forces_order_5_cu).
    Returns f (n,3) [and energy if asked]."""
    assert order == 5
    sz = tuple(int(s) for s in sz)
    L = np.asarray(L, np.float64)
    q = np.asarray(q, np.float64)
    if G is None:
        G = p3m_green(L, sz, alpha, order)
    Qu = math.sqrt(qqr_to_eng)
    ng, d = _p3m_stencil(x, lo, L, sz)
    grid = np.zeros(sz)
    W = [[np.array([_W5(i, d[:, dim]) for i in range(-2, 3)]) for dim in range(3)]][0]
    for a, ix in enumerate(range(-2, 3)):
        px = (ng[:, 0] + ix) % sz[0]
        for b, iy in enumerate(range(-2, 3)):
            py = (ng[:, 1] + iy) % sz[1]
            for c, iz in enumerate(range(-2, 3)):
                pz = (ng[:, 2] + iz) % sz[2]
                w = Qu * q * W[0][a] * W[1][b] * W[2][c]
                np.add.at(grid, (px, py, pz), w)
    rho = np.fft.fftn(grid)
    kx, ky, kz = np.meshgrid(*_kvec(L, sz), indexing="ij")
    V = L[0] * L[1] * L[2]
    E = []
    for k in (kx, ky, kz):
        Ek = 1j * k * rho * G
        E.append(-np.real(np.fft.ifftn(Ek)) * Ek.size / V)
    f = np.zeros((len(x), 3))
    for a, ix in enumerate(range(-2, 3)):
        px = (ng[:, 0] + ix) % sz[0]
        for b, iy in enumerate(range(-2, 3)):
            py = (ng[:, 1] + iy) % sz[1]
            for c, iz in enumerate(range(-2, 3)):
                pz = (ng[:, 2] + iz) % sz[2]
                w = W[0][a] * W[1][b] * W[2][c]
                for dim in range(3):
                    f[:, dim] += w * E[dim][px, py, pz]
    f *= (Qu * q)[:, None]
    if virial is not None:
        # virials_cu + mapVirialToSingleAtom (FixChargeEwald.cu:731-818):
        # 0.5/V sum_k G |rho_k|^2 (delta_ab - 2 (1/k^2 + 1/(4 alpha^2)) k_a k_b), k != 0
        k2 = kx * kx + ky * ky + kz * kz
        Ek = G * np.abs(rho) ** 2
        with np.errstate(divide="ignore", invalid="ignore"):
            dif = np.where(k2 > 0, -2.0 * (1.0 / np.where(k2 > 0, k2, 1.0) + 0.25 / (alpha * alpha)), 0.0)
        Ek = np.where(k2 > 0, Ek, 0.0)
        comps = ((kx, kx, 1.0), (ky, ky, 1.0), (kz, kz, 1.0), (kx, ky, 0.0), (kx, kz, 0.0), (ky, kz, 0.0))
        for c, (ka, kb, dl) in enumerate(comps):
            virial[c] += 0.5 / V * float(np.sum((dl + dif * ka * kb) * Ek))
    if want_energy:
        # 0.5/V sum_k G |rho_k|^2 (FixChargeEwald::singlePointEng, Energy_cu)
        eng = 0.5 / V * float(np.sum(G * np.abs(rho) ** 2))
        return f, eng
    return f


def ewald_recip_direct(x, q, L, alpha, kmax, qqr_to_eng=REAL_UNITS["qqr_to_eng"]):
    """Exact Ewald reciprocal force (sum over |n_i| <= kmax), for pinning P3M."""
    x = np.asarray(x, np.float64)
    q = np.asarray(q, np.float64)
    L = np.asarray(L, np.float64)
    V = np.prod(L)
    f = np.zeros_like(x)
    E = 0.0
    rng = range(-kmax, kmax + 1)
    for nx in rng:
        for ny in rng:
            for nz in rng:
                if nx == 0 and ny == 0 and nz == 0:
                    continue
                k = 2 * math.pi * np.array([nx, ny, nz]) / L
                k2 = k @ k
                A = 4 * math.pi / k2 * math.exp(-k2 / (4 * alpha * alpha))
                ph = x @ k
                S = np.sum(q * np.exp(1j * ph))
                # F_i = -dE/dr_i = -(C/V) A q_i k Im(exp(-i k.r_i) S(k))
                f -= (qqr_to_eng / V * A * q * np.imag(np.exp(-1j * ph) * S))[:, None] * k[None, :]
                E += qqr_to_eng / (2 * V) * A * abs(S) ** 2
    return f, E


# --------------------------------------------------------------------------
# rigid water (FixRigid.cu), FP64
# --------------------------------------------------------------------------
WATER_GEOM = {
    "TIP4P/2005": dict(r_OH=0.9572, r_HH=1.5139, r_OM=0.1546, gamma=0.73612446364836),
    "TIP4P": dict(r_OH=0.9572, r_HH=1.5139, r_OM=0.15, gamma=0.74397533),
    "TIP3P": dict(r_OH=0.9572, r_HH=1.5139, r_OM=0.0, gamma=0.0),
    "SPC": dict(r_OH=1.0, r_HH=1.633, r_OM=0.0, gamma=0.0),
    "SPC/E": dict(r_OH=1.0, r_HH=1.633, r_OM=0.0, gamma=0.0),
}


@dataclass
class RigidData:
    """FixRigidData (FixRigid.h:23-77) as set by setStyleBondLengths,
    set_fixed_sides and populateRigidData (FixRigid.cu:1137-1436)."""
    style: str
    mO: float
    mH: float
    r_OH: float = 0.0
    r_HH: float = 0.0
    r_OM: float = 0.0
    gamma: float = 0.0
    ra: float = 0.0
    rb: float = 0.0
    rc: float = 0.0
    inv2Rc: float = 0.0
    wO: float = 0.0
    wH: float = 0.0
    Minv: np.ndarray = field(default=None)

    def __post_init__(self):
        g = WATER_GEOM[self.style]
        self.r_OH, self.r_HH, self.r_OM, self.gamma = g["r_OH"], g["r_HH"], g["r_OM"], g["gamma"]
        mW = self.mO + 2.0 * self.mH
        self.wO, self.wH = self.mO / mW, self.mH / mW
        rc = 0.5 * self.r_HH
        rab = math.sqrt(self.r_OH ** 2 - rc * rc)
        half = math.atan(rc / rab)
        h1 = 1.5 * math.pi + half
        h2 = 1.5 * math.pi - half
        comy = self.wH * (math.sin(h1) + math.sin(h2)) * self.r_OH
        ra = -comy
        self.ra, self.rb, self.rc, self.inv2Rc = ra, rab - ra, rc, 1.0 / self.r_HH
        inv = self.mO / self.mH
        HH, OH = self.r_HH, self.r_OH
        M = np.array([[1.0 + inv, 1.0 - 0.5 * HH * HH / (OH * OH), inv * 0.5 * HH / OH],
                      [0.0, 0.0, 0.0], [0.0, 0.0, 2.0 * inv]])
        M[1] = [M[0, 1], M[0, 0], M[0, 2]]
        M[2] = [M[0, 2], M[1, 2], 2.0 * inv]
        self.Minv = np.linalg.inv(M) * self.mO


def _mi(v, L):
    return v - L * np.rint(v / L)


def settle_positions(x0, x1, v1, L, rd: RigidData, dt):
    """settlePositions (FixRigid.cu:849-1132), vectorised over molecules.

    x0: (M,3,3) previous constrained O,H1,H2; x1: unconstrained (M,3,3);
    v1: velocities (M,3,3).  Returns new positions and velocities."""
    L = np.asarray(L, np.float64)
    pO0, pH10, pH20 = x0[:, 0], x0[:, 1], x0[:, 2]
    pO, pH1, pH2 = x1[:, 0], x1[:, 1], x1[:, 2]
    b0v = _mi(pH10 - pO0, L)
    c0v = _mi(pH20 - pO0, L)
    oh1 = _mi(pH1 - pO, L)
    oh2 = _mi(pH2 - pO, L)
    pH1 = pO + oh1
    pH2 = pO + oh2
    com = pO + (oh1 + oh2) * rd.wH
    a1 = (oh1 + oh2) * (-rd.wH)
    b1 = pH1 - com
    c1 = pH2 - com
    ax3 = np.cross(b0v, c0v)
    ax1 = np.cross(a1, ax3)
    ax2 = np.cross(ax3, ax1)
    ax1 /= np.linalg.norm(ax1, axis=1)[:, None]
    ax2 /= np.linalg.norm(ax2, axis=1)[:, None]
    ax3 /= np.linalg.norm(ax3, axis=1)[:, None]

    def rot(v):
        return np.stack([np.sum(ax1 * v, 1), np.sum(ax2 * v, 1), np.sum(ax3 * v, 1)], 1)

    rb0, rc0 = rot(b0v), rot(c0v)
    ra1, rb1, rc1 = rot(a1), rot(b1), rot(c1)
    ra, rb, rc = rd.ra, rd.rb, rd.rc
    sinPhi = ra1[:, 2] / ra
    cosPhi = np.sqrt(1.0 - sinPhi * sinPhi)
    sinPsi = (rb1[:, 2] - rc1[:, 2]) * (rd.inv2Rc / cosPhi)
    cosPsi = np.sqrt(1.0 - sinPsi * sinPsi)
    a2 = np.stack([np.zeros_like(cosPhi), ra * cosPhi, rb * sinPhi], 1)
    b2 = np.stack([-rc * cosPsi, -rb * cosPhi - rc * sinPsi * sinPhi, -rb * sinPhi + rc * sinPsi * cosPhi], 1)
    c2 = np.stack([rc * cosPsi, -rb * cosPhi + rc * sinPsi * sinPhi, -rb * sinPhi - rc * sinPsi * cosPhi], 1)
    alpha = b2[:, 0] * (rb0[:, 0] - rc0[:, 0]) + b2[:, 1] * rb0[:, 1] + c2[:, 1] * rc0[:, 1]
    beta = b2[:, 0] * (rc0[:, 1] - rb0[:, 1]) + b2[:, 1] * rb0[:, 0] + c2[:, 1] * rc0[:, 0]
    gamma = rb0[:, 0] * rb1[:, 1] - rb1[:, 0] * rb0[:, 1] + rc0[:, 0] * rc1[:, 1] - rc1[:, 0] * rc0[:, 1]
    a2b2 = alpha * alpha + beta * beta
    sinT = (alpha * gamma - beta * np.sqrt(a2b2 - gamma * gamma)) / a2b2
    cosT = np.sqrt(1.0 - sinT * sinT)
    a3 = np.stack([-a2[:, 1] * sinT, a2[:, 1] * cosT, ra1[:, 2]], 1)
    b3 = np.stack([b2[:, 0] * cosT - b2[:, 1] * sinT, b2[:, 0] * sinT + b2[:, 1] * cosT, b2[:, 2]], 1)
    c3 = np.stack([c2[:, 0] * cosT - c2[:, 1] * sinT, c2[:, 0] * sinT + c2[:, 1] * cosT, c2[:, 2]], 1)

    def back(v):
        return ax1 * v[:, 0:1] + ax2 * v[:, 1:2] + ax3 * v[:, 2:3]

    ap, bp, cp = back(a3), back(b3), back(c3)
    xn = np.stack([ap + com, bp + com, cp + com], 1)
    invdt = 1.0 / dt
    vn = v1.copy()
    vn[:, 0] += (ap - a1) * invdt
    vn[:, 1] += (bp - b1) * invdt
    vn[:, 2] += (cp - c1) * invdt
    return xn, vn


def settle_velocities(x, v, L, rd: RigidData):
    """settleVelocities (FixRigid.cu:657-846): x (M,3,3) constrained positions."""
    L = np.asarray(L, np.float64)
    rOH1 = _mi(x[:, 0] - x[:, 1], L) / rd.r_OH
    rOH2 = _mi(x[:, 0] - x[:, 2], L) / rd.r_OH
    rHH = _mi(x[:, 1] - x[:, 2], L) / rd.r_HH
    rel = np.stack([np.sum((v[:, 0] - v[:, 1]) * rOH1, 1), np.sum((v[:, 0] - v[:, 2]) * rOH2, 1),
                    np.sum((v[:, 1] - v[:, 2]) * rHH, 1)], 1)
    vc = rel @ rd.Minv.T
    vn = v.copy()
    vn[:, 0] += (rOH1 * vc[:, 0:1] + rOH2 * vc[:, 1:2]) * (-1.0 / rd.mO)
    vn[:, 1] += (-rOH1 * vc[:, 0:1] + rHH * vc[:, 2:3]) * (-1.0 / rd.mH)
    vn[:, 2] += (-rOH2 * vc[:, 1:2] - rHH * vc[:, 2:3]) * (-1.0 / rd.mH)
    return vn


def msite_positions(xO, xH1, xH2, L, r_OM):
    """setMSite (FixRigid.cu:560-599)."""
    L = np.asarray(L, np.float64)
    rij = _mi(xH1 - xO, L)
    rik = _mi(xH2 - xO, L)
    s = rij + rik
    return xO + r_OM * s / np.linalg.norm(s, axis=1)[:, None]


def msite_distribute(fO, fH1, fH2, fM, vO, vH1, vH2, invmO, invmH, gamma, dtf):
    """distributeMSite<FORCES> (FixRigid.cu:475-558)."""
    fOd = fM * gamma
    fHd = fM * 0.5 * (1.0 - gamma)
    return (fO + fOd, fH1 + fHd, fH2 + fHd,
            vO + dtf * invmO * fOd, vH1 + dtf * invmH * fHd, vH2 + dtf * invmH * fHd)


# --------------------------------------------------------------------------
# Nose-Hoover chain (FixNoseHoover.cu), host FP64 exactly as the reference
# --------------------------------------------------------------------------
class NoseHooverChain:
    """FixNoseHoover's particle chain (FixNoseHoover.cu:221-290, 795-866,
    1034-1041) in FP64, the library's precision.  ref_float: in the
    reference's own precision instead -- its frequency and kinetic energy
    are floats (`real frequency`, `real ke_current`, FixNoseHoover.h), as
    are its time step (State.h:117) and Boltzmann constant (Units.h:8), and
    M v^2 is taken as (M v) v.  Pinned against the reference's own chain
    compiled from source on the CPU (oracle/ref_nh_harness.cu): bit for bit
    with ref_float, to 1e-5 in FP64 over 40 steps."""

    def __init__(self, T, tau, ndf, boltz, dt, chain=10, ref_float=False):
        self.rf = ref_float
        if ref_float:
            f32 = np.float32
            self.freq, boltz, dt = float(f32(1.0 / tau)), float(f32(boltz)), float(f32(dt))
        else:
            self.freq = 1.0 / tau
        self.T, self.ndf, self.kB, self.dt = T, ndf, boltz, dt
        self.n = chain
        self.vel = [0.0] * chain
        self.force = [0.0] * chain
        self.mass = [0.0] * chain
        self.ke = 0.0
        self.scale = 1.0

    def _freq2(self):
        if self.rf:
            return float(np.float32(self.freq) * np.float32(self.freq))
        return self.freq ** 2

    def _mv2(self, m, v):
        return m * v * v if self.rf else m * v ** 2

    def update_masses(self):
        f2 = self._freq2()
        self.mass[0] = self.ndf * self.kB * self.T / f2
        for i in range(1, self.n):
            self.mass[i] = self.kB * self.T / f2

    def prepare(self, ke):
        """prepareFinal (FixNoseHoover.cu:240-290): ke = sum m v^2 * mvv_to_eng."""
        self.ke = float(np.float32(ke)) if self.rf else ke
        self.update_masses()
        self.force[0] = (self.ke - self.ndf * self.kB * self.T) / self.mass[0]
        for k in range(1, self.n):
            self.force[k] = (self._mv2(self.mass[k - 1], self.vel[k - 1]) - self.kB * self.T) / self.mass[k]

    def integrate(self, step_init):
        """thermostatIntegrate (FixNoseHoover.cu:795-866); returns the
        velocity scale factor accumulated in this call."""
        nkt = self.ndf * self.kB * self.T
        if not step_init:
            self.force[0] = (self.ke - nkt) / self.mass[0]
        ts = self.dt
        t2, t4, t8 = 0.5 * ts, 0.25 * ts, 0.125 * ts
        v, F, Q = self.vel, self.force, self.mass
        n = self.n
        v[n - 1] += t4 * F[n - 1]
        for k in range(n - 2, 0, -1):
            pf = math.exp(-t8 * v[k + 1])
            v[k] *= pf
            v[k] += t4 * F[k]
            v[k] *= pf
        pf = math.exp(-t8 * v[1])
        v[0] *= pf
        v[0] += t4 * F[0]
        v[0] *= pf
        sf = math.exp(-t2 * v[0])
        if self.rf:
            self.ke = float(np.float32(self.ke * (sf * sf)))
        else:
            self.ke *= sf * sf
        v[0] *= pf
        F[0] = (self.ke - nkt) / Q[0]
        v[0] += t4 * F[0]
        v[0] *= pf
        for k in range(1, n - 1):
            pf = math.exp(-t8 * v[k + 1])
            v[k] *= pf
            F[k] = (self._mv2(Q[k - 1], v[k - 1]) - self.kB * self.T) / Q[k]
            v[k] += t4 * F[k]
            v[k] *= pf
        F[n - 1] = (self._mv2(Q[n - 2], v[n - 2]) - self.kB * self.T) / Q[n - 1]
        v[n - 1] += t4 * F[n - 1]
        return sf


def kinetic_sum(v, invm):
    """sum m v^2 over atoms with finite mass (SumVectorSqr3DOverW, cutils_func.h)."""
    ok = invm < 1e18
    return float(np.sum(np.sum(v[ok] ** 2, 1) / invm[ok]))
