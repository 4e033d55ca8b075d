"""ctypes access to the reference's own kernels compiled from source
(oracle/ref.mk -> oracle/_ref/librefkernels.so) -- TEST INFRASTRUCTURE ONLY.
Used by the GPU parity tests to run the reference kernels on the same GPU and
inputs as the B200 kernels.  Absent when the reference sources were not
mounted at build time; callers skip then."""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
PATH = os.path.join(_HERE, "_ref", "librefkernels.so")
_L = None


def available():
    return os.path.exists(PATH)


def lib():
    global _L
    if _L is None:
        _L = ctypes.CDLL(PATH)
        V = ctypes.c_void_p
        I = ctypes.c_int
        F = ctypes.c_float
        _L.ref_pair_forces.argtypes = [I, V, V, V, V, I, V, I, V, V, F, F, F, I, F, F, F, I, I, V]
        _L.ref_pair_forces.restype = I
        _L.ref_e3b_forces.argtypes = [I, V, I, V, V, V, I, V, V, I, I, I, V]
        _L.ref_e3b_forces.restype = I
        _L.ref_set_timing.argtypes = [I]
        _L.ref_last_ms.restype = F
        _L.ref_lj_force_host.argtypes = [F, F, F, V, V]
        _L.ref_e3b_single_host.argtypes = [F, V]
        _L.ref_ljfs_host.argtypes = [F, F, F, V, V]
        _L.ref_pair_styles.argtypes = [I, V, V, V, V, I, V, I, I, V, V, F, F, F, I, I, F, F, F, F, F, I, I, V]
        _L.ref_pair_styles.restype = I
        _L.ref_grid_skin_flag.argtypes = [I, V, V, V, V, F]
        _L.ref_grid_skin_flag.restype = I
        _L.ref_grid_build.argtypes = [I, V, V, V, V, F, I, I, I, V, V, V]
        _L.ref_grid_build.restype = I
        D = ctypes.c_double
        _L.ref_settle.argtypes = [I, V, V, V, V, V, V, D, D, I]
        _L.ref_settle.restype = I
    return _L


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def pair_forces(xs4, q, counts, nbr, params_flat, ntypes, lo, L, coef, lj_kind, qcut, alpha, qqr,
                ntpb=256, ntpa=8):
    xs4 = np.ascontiguousarray(xs4, np.float32)
    n = len(xs4)
    q = np.ascontiguousarray(q if q is not None else np.zeros(n), np.float32)
    counts = np.ascontiguousarray(counts, np.int32)
    nbr = np.ascontiguousarray(nbr, np.uint32)
    pf = np.ascontiguousarray(params_flat, np.float32)
    lo = np.ascontiguousarray(lo, np.float32)
    L = np.ascontiguousarray(L, np.float32)
    out = np.zeros((n, 4), np.float32)
    rc = lib().ref_pair_forces(n, _p(xs4), _p(q), _p(counts), _p(nbr), nbr.shape[1], _p(pf), ntypes, _p(lo), _p(L),
                               coef[0], coef[1], coef[2], lj_kind, qcut, alpha, qqr, ntpb, ntpa, _p(out))
    if rc != 0:
        raise RuntimeError(f"reference pair kernel failed: {rc}")
    return out[:, :3].astype(np.float64)


def pair_styles(xs4, q, counts, nbr, table, ntypes, lo, L, coef, lj_kind, ck, qcut=0.0, alpha=0.0, qqr=1.0,
                dsf_A=0.0, dsf_shift=0.0, ntpb=256, ntpa=8):
    """the reference's compute_force_iso with EvaluatorLJFS (lj_kind 3),
    EvaluatorCHARMM (4), EvaluatorTICG (5) or EvaluatorLJ (1, with DSF) and
    ChargeEvaluatorNone / Ewald / DSF (ck 0 / 1 / 2); table: np x nt x nt"""
    xs4 = np.ascontiguousarray(xs4, np.float32)
    n = len(xs4)
    q = np.ascontiguousarray(q if q is not None else np.zeros(n), np.float32)
    counts = np.ascontiguousarray(counts, np.int32)
    nbr = np.ascontiguousarray(nbr, np.uint32)
    tb = np.ascontiguousarray(table, np.float32)
    lo = np.ascontiguousarray(lo, np.float32)
    L = np.ascontiguousarray(L, np.float32)
    out = np.zeros((n, 4), np.float32)
    rc = lib().ref_pair_styles(n, _p(xs4), _p(q), _p(counts), _p(nbr), nbr.shape[1], _p(tb), tb.shape[0], ntypes,
                               _p(lo), _p(L), coef[0], coef[1], coef[2], lj_kind, ck, qcut, alpha, qqr, dsf_A,
                               dsf_shift, ntpb, ntpa, _p(out))
    if rc != 0:
        raise RuntimeError(f"reference pair kernel failed: {rc}")
    return out[:, :3].astype(np.float64)


def ljfs_host(sigma, eps, rcut, dr):
    d = np.ascontiguousarray(dr, np.float32)
    o = np.zeros(4, np.float32)
    lib().ref_ljfs_host(sigma, eps, rcut, _p(d), _p(o))
    return o


def e3b_forces(xs4, mol, mcounts, mnbr, lo, L, style3=True, ntpb=256, ntpa=8):
    xs4 = np.ascontiguousarray(xs4, np.float32)
    mol = np.ascontiguousarray(mol, np.int32)
    mcounts = np.ascontiguousarray(mcounts, np.int32)
    mnbr = np.ascontiguousarray(mnbr, np.uint32)
    lo = np.ascontiguousarray(lo, np.float32)
    L = np.ascontiguousarray(L, np.float32)
    out = np.zeros((len(xs4), 4), np.float32)
    rc = lib().ref_e3b_forces(len(xs4), _p(xs4), len(mol), _p(mol), _p(mcounts), _p(mnbr), mnbr.shape[1], _p(lo),
                              _p(L), 1 if style3 else 0, ntpb, ntpa, _p(out))
    if rc != 0:
        raise RuntimeError(f"reference E3B kernels failed: {rc}")
    return out[:, :3].astype(np.float64)


def lj_force_host(sigma, eps, rcut, dr):
    d = np.ascontiguousarray(dr, np.float32)
    o = np.zeros(3, np.float32)
    lib().ref_lj_force_host(sigma, eps, rcut, _p(d), _p(o))
    return o


def e3b_single_host(r):
    o = np.zeros(4, np.float32)
    lib().ref_e3b_single_host(float(r), _p(o))
    return o


def timed(fn, iters, *a, **kw):
    """run fn (pair_forces / e3b_forces) once for its result, then its
    launch(es) `iters` more times between CUDA events: (result, mean ms)"""
    lib().ref_set_timing(int(iters))
    try:
        out = fn(*a, **kw)
        return out, float(lib().ref_last_ms())
    finally:
        lib().ref_set_timing(0)


def grid_skin_flag(xa, xb, lo, L, padding):
    """the reference's setBuildFlag on positions xa (current) and xb (last
    build): 1 if some atom moved more than padding / 2"""
    a = np.zeros((len(xa), 4), np.float32)
    a[:, :3] = xa
    b = np.zeros((len(xb), 4), np.float32)
    b[:, :3] = xb
    lo = np.ascontiguousarray(lo, np.float32)
    L = np.ascontiguousarray(L, np.float32)
    r = lib().ref_grid_skin_flag(len(a), _p(a), _p(b), _p(lo), _p(L), float(padding))
    if r < 0:
        raise RuntimeError(f"reference setBuildFlag failed: {r}")
    return r


def grid_build(x, lo, L, neigh_cut, min_dim=None, ntpb=256, ntpa=1, maxn=512):
    """a forced build of the reference's GridGPU kernels on positions x (ids
    0..n-1): per id its neighbour count, its neighbours' ids (list order) and
    the wrapped position the list was built on"""
    n = len(x)
    xs4 = np.zeros((n, 4), np.float32)
    xs4[:, :3] = x
    lo = np.ascontiguousarray(lo, np.float32)
    L = np.ascontiguousarray(L, np.float32)
    md = np.ascontiguousarray(min_dim if min_dim is not None else np.full(3, neigh_cut), np.float32)
    counts = np.zeros(n, np.int32)
    nbr = np.zeros((n, maxn), np.uint32)
    wrapped = np.zeros((n, 4), np.float32)
    r = lib().ref_grid_build(n, _p(xs4), _p(lo), _p(L), _p(md), float(neigh_cut), ntpb, ntpa, maxn, _p(counts),
                             _p(nbr), _p(wrapped))
    if r != 0:
        raise RuntimeError(f"reference GridGPU build failed: {r}")
    return counts, nbr, wrapped[:, :3]


def settle(x0, x, v, masses, lo, L, dt, ftm_to_v, mode):
    """the reference's SETTLE on rigid TIP4P/2005 molecules laid out O, H1,
    H2, M per molecule (n = 4 * nmol sites): mode 1 settles the positions x
    (from the constrained x0 of the step's start) and velocities v, then
    places M (settlePositions + setMSite); mode 2 settles the velocities v at
    the positions x (settleVelocities).  Returns (x, v) as float64."""
    n = len(x)
    def four(a, w=None):
        o = np.zeros((n, 4), np.float32)
        o[:, :3] = a
        if w is not None:
            o[:, 3] = w
        return o
    X0, X, Vv = four(x0), four(x), four(v)
    ms = np.ascontiguousarray(masses, np.float64)
    lo = np.ascontiguousarray(lo, np.float32)
    L = np.ascontiguousarray(L, np.float32)
    r = lib().ref_settle(n // 4, _p(X0), _p(X), _p(Vv), _p(ms), _p(lo), _p(L), float(dt), float(ftm_to_v), mode)
    if r != 0:
        raise RuntimeError(f"reference SETTLE failed: {r}")
    return X[:, :3].astype(np.float64), Vv[:, :3].astype(np.float64)


BAROSTAT_PATH = os.path.join(_HERE, "_ref", "librefbarostat.so")
_NH = None


def barostat_available():
    return os.path.exists(BAROSTAT_PATH)


def _barostat_lib():
    global _NH
    if _NH is None:
        _NH = ctypes.CDLL(BAROSTAT_PATH)
        V = ctypes.c_void_p
        I = ctypes.c_int
        D = ctypes.c_double
        _NH.ref_nh_barostat.argtypes = [I, I, V, I, V, V, V, V, V]
        _NH.ref_nh_barostat.restype = I
        _NH.ref_berendsen_dilation.argtypes = [D, D, D, D, D, D, V]
        _NH.ref_berendsen_dilation.restype = I
        _NH.ref_nh_chain.argtypes = [I, I, V, I, V, V, V, V, V]
        _NH.ref_nh_chain.restype = I
    return _NH


def nh_barostat(op, step_init, par, pvel, pmass, ptv, ptf, ptm):
    """one call of the reference's host-side isotropic MTK propagator
    (FixNoseHoover.cu compiled from source into oracle/_ref/librefbarostat.so;
    no GPU needed): op 0 updateBarostatMasses, 1 updateBarostatThermalMasses,
    2 barostatThermostatIntegrate, 3 barostatVelocityIntegrate.  par = (natoms,
    ndf, T, P, pfreq, dt, boltz, nktv_to_press, p_inst, t_inst, Lx, Ly, Lz).
    Returns the updated (pvel, pmass, ptv, ptf, ptm) as new float64 arrays."""
    par = np.ascontiguousarray(par, np.float64)
    assert par.shape == (13,)
    out = [np.array(a, np.float64, copy=True) for a in (pvel, pmass, ptv, ptf, ptm)]
    chain = len(out[2])
    assert len(out[0]) == len(out[1]) == 3 and len(out[3]) == len(out[4]) == chain
    r = _barostat_lib().ref_nh_barostat(int(op), int(bool(step_init)), _p(par), chain, *(_p(a) for a in out))
    if r != 0:
        raise RuntimeError(f"reference barostat propagator failed: {r}")
    return tuple(out)


def berendsen_dilation(target, pressure, period, dt, bulk=-1.0, max_dil=-1.0):
    """the box scale factors of one reference FixPressureBerendsen step
    (stepFinal, FixPressureBerendsen.cu:26-46, compiled from source into
    oracle/_ref/librefbarostat.so; no GPU needed) at the instantaneous
    pressure `pressure`; bulk / max_dil < 0 keep the fix's defaults.
    Returns the three float32 factors."""
    out = np.zeros(3, np.float32)
    r = _barostat_lib().ref_berendsen_dilation(float(target), float(pressure), float(period), float(dt),
                                               float(bulk), float(max_dil), _p(out))
    if r != 0:
        raise RuntimeError(f"reference Berendsen step failed: {r}")
    return out


def nh_chain(op, step_init, par, tvel, tforce, tmass, ke, scale):
    """one call on the reference's particle Nose-Hoover chain of a
    thermostat-only FixNoseHoover (compiled from source into
    oracle/_ref/librefbarostat.so; no GPU needed): op 0 prepareFinal, 1
    updateThermalMasses, 2 thermostatIntegrate.  par = (natoms, ndf, T, tau,
    dt, boltz).  Returns the updated (tvel, tforce, tmass) as new float64
    arrays and the kinetic energy and velocity scale (float-rounded, as the
    fix holds them)."""
    par = np.ascontiguousarray(par, np.float64)
    assert par.shape == (6,)
    out = [np.array(a, np.float64, copy=True) for a in (tvel, tforce, tmass)]
    assert len(out[0]) == len(out[1]) == len(out[2])
    kes = np.array([ke, scale], np.float64)
    r = _barostat_lib().ref_nh_chain(int(op), int(bool(step_init)), _p(par), len(out[0]), *(_p(a) for a in out),
                                     _p(kes[0:]), _p(kes[1:]))
    if r != 0:
        raise RuntimeError(f"reference Nose-Hoover chain failed: {r}")
    return out[0], out[1], out[2], float(kes[0]), float(kes[1])


EWALD_PATH = os.path.join(_HERE, "_ref", "librefewald.so")
_EW = None


def ewald_available():
    return os.path.exists(EWALD_PATH)


def _ewald_lib():
    global _EW
    if _EW is None:
        _EW = ctypes.CDLL(EWALD_PATH)
        V = ctypes.c_void_p
        I = ctypes.c_int
        D = ctypes.c_double
        _EW.ref_ewald_alpha.argtypes = [I, V, V, D, I, D, V, V]
        _EW.ref_ewald_alpha.restype = I
        _EW.ref_ewald_green.argtypes = [V, V, D, I, V]
        _EW.ref_ewald_green.restype = I
    return _EW


def ewald_alpha(natoms, L, sz, rcut, order, q2):
    """the reference's FixChargeEwald::find_optimal_parameters
    (FixChargeEwald.cu:918-967, compiled from source into
    oracle/_ref/librefewald.so; host code, run where a GPU is) for natoms
    atoms in a box of sides L, mesh sz, cutoff rcut, interpolation order
    `order`, total squared charge q2 (times qqr_to_eng).  Returns (alpha, the
    RMS error estimate); alpha is the float the fix keeps."""
    Ld = np.ascontiguousarray(L, np.float64)
    szi = np.ascontiguousarray(sz, np.int32)
    out = np.zeros(2, np.float64)
    r = _ewald_lib().ref_ewald_alpha(int(natoms), _p(Ld), _p(szi), float(rcut), int(order), float(q2), _p(out[0:]),
                                     _p(out[1:]))
    if r != 0:
        raise RuntimeError(f"reference Ewald parameter solve failed: {r}")
    return float(out[0]), float(out[1])


def ewald_green(L, sz, alpha, order):
    """the reference's influence function (Green_function_cu,
    FixChargeEwald.cu:314-366, launched by calc_Green_function on the GPU)
    for a box of sides L, mesh sz, splitting parameter alpha and
    interpolation order `order`: float32 array of shape sz."""
    Ld = np.ascontiguousarray(L, np.float64)
    szi = np.ascontiguousarray(sz, np.int32)
    out = np.zeros(tuple(int(x) for x in sz), np.float32)
    r = _ewald_lib().ref_ewald_green(_p(Ld), _p(szi), float(alpha), int(order), _p(out))
    if r != 0:
        raise RuntimeError(f"reference Green function failed: {r}")
    return out
