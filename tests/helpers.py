"""Shared set-up for the parity tests: the same seeded systems go through the
CUDA path (via the C ABI) and the CPU oracle."""
from __future__ import annotations

import numpy as np

from md_engine_b200 import systems

# Force tolerance used by every FP32-vs-FP64 force comparison: the largest
# per-atom error vector, relative to the RMS force of the system.
FORCE_RTOL = 2e-4


def water_small(nside=8, seed=11):
    """512-molecule box (L = 24.9 A) for parity tests: rc 6.5, skin 1.0."""
    return systems.water_tip4p2005(nside=nside, seed=seed)


def f32(x):
    return np.asarray(x, np.float32).astype(np.float64)


def force_err(f_gpu, f_ref):
    rms = np.sqrt(np.mean(np.sum(f_ref ** 2, 1)))
    err = np.max(np.linalg.norm(f_gpu - f_ref, axis=1))
    return err / rms, rms


def oracle_lj_params(O, sysd, rcut, wca=False):
    nt = len(sysd.species)
    return O.lj_params(nt, {(0, 0): 1.0}, {(0, 0): 1.0}, rcut, wca=wca)


def oracle_water_params(O, rcut):
    sig = {(0, 0): systems.SIG_OO, (1, 1): 0.0, (0, 1): 0.0, (2, 2): 0.0}
    eps = {(0, 0): systems.EPS_OO, (1, 1): 0.0, (0, 1): 0.0, (2, 2): 0.0}
    return O.lj_params(3, sig, eps, rcut)


def water_bonds(mol):
    b = []
    for o, h1, h2, m in mol:
        b += [(o, h1), (o, h2), (h1, h2), (o, m)]
    return b


def oracle_nlist_for(O, x_wrapped_f32, lo, L, cut, ids=None, excl=None):
    xs4 = np.zeros((len(x_wrapped_f32), 4), np.float32)
    xs4[:, :3] = x_wrapped_f32
    return O.nlist_cells(xs4, lo, L, cut, ids=ids, excl=excl)


def neighbor_cut(rcut, padding):
    """neighCut as GridGPU builds it: (float)((double)(float)rCut + padding)."""
    return np.float32(float(np.float32(rcut)) + padding)
