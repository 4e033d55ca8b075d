"""Seeded synthetic systems of the benchmark shapes, and builders that set up
a State the way the reference's scripts do (benchmark/benchmark.py,
examples/e3b3_speed/e3b3_4000.py, util_py/water.py:196-233).

No dataset or reference file is read: positions come from lattices, water
orientations from seeded uniform random rotations, velocities from seeded
Maxwell-Boltzmann draws with zero total momentum, rescaled to the target T.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

DEFAULT_SEED = 20261203

# TIP4P/2005 (util_py/water.py:196-198, FixRigid.cu:1371-1379)
QH = 0.5564
QM = -2.0 * QH
R_OH = 0.9572
R_HH = 1.5139
R_OM = 0.1546
MASS_O = 15.9994
MASS_H = 1.008
SIG_OO = 3.1589
EPS_OO = 0.185207422
WATER_MOLAR_MASS = 18.01528
AVOGADRO = 6.02214076e23
BOLTZ_REAL = 0.0019872067
MVV_TO_ENG_REAL = 48.88821291 * 48.88821291


@dataclass
class System:
    pos: np.ndarray        # (n,3) float64
    vel: np.ndarray        # (n,3)
    types: np.ndarray      # (n,) int
    q: np.ndarray          # (n,)
    mass: np.ndarray       # (n,)
    L: np.ndarray          # (3,)
    lo: np.ndarray         # (3,)
    species: list          # [(handle, mass, atomicNum)]
    molecules: np.ndarray  # (M,4) ids O,H1,H2,M or empty


def _mb_velocities(rng, mass, T, kB, mvv):
    """Maxwell-Boltzmann draw with zero momentum, exactly rescaled to T
    (InitializeAtoms::initTemp, InitializeAtoms.cpp:98-130)."""
    n = len(mass)
    v = np.zeros((n, 3))
    ok = mass > 0
    v[ok] = rng.standard_normal((ok.sum(), 3)) * np.sqrt(1.0 / mass[ok])[:, None]
    mtot = mass[ok].sum()
    p = (v[ok] * mass[ok][:, None]).sum(0)
    v[ok] -= p / mtot
    ke2 = float((mass[ok][:, None] * v[ok] ** 2).sum()) * mvv
    ndf = 3 * ok.sum()
    v[ok] *= math.sqrt(ndf * kB * T / ke2)
    return v


def lj_fcc(ncell=20, rho=0.8442, T=1.2, seed=DEFAULT_SEED, jitter=0.0):
    """LJ fluid: 4*ncell^3 atoms on an FCC lattice at reduced density rho
    (optionally displaced by a seeded normal jitter of `jitter` sigma)."""
    a = (4.0 / rho) ** (1.0 / 3.0)
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    g = np.stack(np.meshgrid(np.arange(ncell), np.arange(ncell), np.arange(ncell), indexing="ij"), -1).reshape(-1, 3)
    pos = ((g[:, None, :] + base[None, :, :]).reshape(-1, 3) + 0.25) * a
    n = len(pos)
    rng = np.random.default_rng(seed)
    if jitter:
        pos = pos + rng.normal(0.0, jitter, pos.shape)
    mass = np.ones(n)
    vel = _mb_velocities(rng, mass, T, 1.0, 1.0)
    L = np.full(3, ncell * a)
    return System(pos, vel, np.zeros(n, int), np.zeros(n), mass, L, np.zeros(3), [("A", 1.0, 1)],
                  np.zeros((0, 4), int))


def _random_rotations(rng, m):
    q = rng.standard_normal((m, 4))
    q /= np.linalg.norm(q, axis=1)[:, None]
    w, x, y, z = q.T
    R = np.empty((m, 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z)
    R[:, 0, 1] = 2 * (x * y - z * w)
    R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w)
    R[:, 1, 1] = 1 - 2 * (x * x + z * z)
    R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w)
    R[:, 2, 1] = 2 * (y * z + x * w)
    R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


def water_tip4p2005(nside=16, density=0.997, T=298.0, seed=DEFAULT_SEED, nmol=None):
    """nside^3 rigid TIP4P/2005 molecules on a cubic lattice at `density`
    g/cm^3 with seeded random orientations; ids per molecule O, H1, H2, M.
    With nmol, a box for nmol molecules at that density whose lattice of
    ceil(nmol^(1/3))^3 sites is filled at nmol seeded random sites."""
    m = nside ** 3 if nmol is None else int(nmol)
    if nmol is not None:
        nside = int(math.ceil(m ** (1.0 / 3.0) - 1e-9))
    vol_per = WATER_MOLAR_MASS / (density * AVOGADRO) * 1e24  # A^3
    L = (m * vol_per) ** (1.0 / 3.0)
    sp = L / nside
    g = np.stack(np.meshgrid(np.arange(nside), np.arange(nside), np.arange(nside), indexing="ij"), -1).reshape(-1, 3)
    if nmol is not None:
        pick = np.sort(np.random.default_rng(seed + 1).choice(len(g), m, replace=False))
        g = g[pick]
    centers = (g + 0.5) * sp
    half = math.asin(0.5 * R_HH / R_OH)
    local = np.array([
        [0.0, 0.0, 0.0],
        [R_OH * math.sin(half), R_OH * math.cos(half), 0.0],
        [-R_OH * math.sin(half), R_OH * math.cos(half), 0.0],
        [0.0, R_OM, 0.0],
    ])
    rng = np.random.default_rng(seed)
    R = _random_rotations(rng, m)
    pos = centers[:, None, :] + np.einsum("mij,kj->mki", R, local)
    pos = pos.reshape(-1, 3)
    types = np.tile([0, 1, 1, 2], m)
    q = np.tile([0.0, QH, QH, QM], m)
    mass = np.tile([MASS_O, MASS_H, MASS_H, 0.0], m)
    vel = _mb_velocities(rng, mass, T, BOLTZ_REAL, MVV_TO_ENG_REAL)
    mol = np.arange(4 * m).reshape(m, 4)
    species = [("OW", MASS_O, 8), ("HY", MASS_H, 1), ("OM", 0.0, 0)]
    return System(pos, vel, types, q, mass, np.full(3, L), np.zeros(3), species, mol)


def build_lj_state(sysd: System, rcut=2.5, skin=0.3, dt=0.005, interval=10, T=None, tau=None, wca=False):
    """LJ fluid state as benchmark/benchmark.py (LJ units)."""
    from .dash import Bounds, FixLJCut, FixNoseHoover, FixWCA, State, Vector
    st = State()
    st.units.setLJ()
    st.bounds = Bounds(st, lo=Vector(*sysd.lo), hi=Vector(*(sysd.lo + sysd.L)))
    st.rCut = rcut
    st.padding = skin
    st.dt = dt
    st.periodicInterval = interval
    for h, mm, z in sysd.species:
        st.atomParams.addSpecies(handle=h, mass=mm, atomicNum=z)
    handles = [sysd.species[t][0] for t in sysd.types]
    st.addAtoms(handles, sysd.pos, sysd.q)
    st.setVelocities(np.arange(len(sysd.pos)), sysd.vel)
    fixes = []
    pair = (FixWCA if wca else FixLJCut)(st, "wca" if wca else "ljcut")
    pair.setParameter("sig", "A", "A", 1.0)
    pair.setParameter("eps", "A", "A", 1.0)
    st.activateFix(pair)
    fixes.append(pair)
    if T is not None:
        nh = FixNoseHoover(st, "nvt", "all")
        nh.setTemperature(T, tau)
        st.activateFix(nh)
        fixes.append(nh)
    return st, fixes


def build_water_state(sysd: System, rcut=9.0, skin=1.0, dt=2.0, interval=10, grid=64, e3b=False,
                      T=298.0, tau=100.0, alpha=None, thermostat=True):
    """Rigid TIP4P/2005 (+ optional E3B3) state as examples/e3b3_speed/e3b3_4000.py."""
    from .dash import (Bounds, FixChargeEwald, FixE3B, FixLJCut, FixNoseHoover, FixRigid, State, Vector)
    st = State()
    st.units.setReal()
    st.bounds = Bounds(st, lo=Vector(*sysd.lo), hi=Vector(*(sysd.lo + sysd.L)))
    st.rCut = rcut
    st.padding = skin
    st.dt = dt
    st.periodicInterval = interval
    for h, mm, z in sysd.species:
        st.atomParams.addSpecies(handle=h, mass=mm, atomicNum=z)
    handles = [sysd.species[t][0] for t in sysd.types]
    st.addAtoms(handles, sysd.pos, sysd.q)
    st.setVelocities(np.arange(len(sysd.pos)), sysd.vel)
    lj = FixLJCut(st, "cut")
    lj.setParameter("sig", "OW", "OW", SIG_OO)
    lj.setParameter("eps", "OW", "OW", EPS_OO)
    for a, b in (("HY", "HY"), ("OW", "HY"), ("OM", "OM")):
        lj.setParameter("sig", a, b, 0.0)
        lj.setParameter("eps", a, b, 0.0)
    ew = FixChargeEwald(st, "charge", "all")
    ew.setParameters(grid, grid, grid, rcut, 5)
    if alpha is not None:
        ew.setAlpha(alpha)
    rigid = FixRigid(st, "rigid", "TIP4P/2005")
    for o, h1, h2, mm in sysd.molecules:
        rigid.createRigid(o, h1, h2, mm)
    fixes = {"lj": lj, "ewald": ew, "rigid": rigid}
    st.activateFix(lj)
    st.activateFix(ew)
    st.activateFix(rigid)
    if e3b:
        f3 = FixE3B(st, "e3b3", "E3B3")
        for o, h1, h2, mm in sysd.molecules:
            f3.addMolecule(o, h1, h2, mm)
        st.activateFix(f3)
        fixes["e3b"] = f3
    if thermostat:
        nh = FixNoseHoover(st, "nvt", "all")
        nh.setTemperature(T, tau)
        st.activateFix(nh)
        fixes["nh"] = nh
    return st, fixes


def water_replica_sizes(nrep=64, lo=256, hi=2048, seed=DEFAULT_SEED):
    """molecule counts drawn log-uniform in [lo, hi] and temperatures uniform
    in [260, 360] K, seeded (the batched-replica workload)"""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(math.log(lo), math.log(hi), nrep)).round().astype(int)
    temps = rng.uniform(260.0, 360.0, nrep)
    return sizes, temps


def p3m_mesh_for(L, h_max=1.0):
    """smallest power-of-two mesh with spacing <= h_max (the 2^N rule of the
    reference's examples)"""
    n = 8
    while L / n > h_max:
        n *= 2
    return n
