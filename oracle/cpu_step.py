"""Whole-timestep CPU oracle -- TEST AND CPU-BASELINE INFRASTRUCTURE ONLY.

Composes the oracle's FP64 restatements in the reference's hook order
(IntegratorVerlet.cu:694-754): Nose-Hoover stepInit -> save_prev -> nve_v/x
-> SETTLE positions + M sites -> neighbour list + pair forces (LJ + Ewald
real) + P3M (+ E3B) -> postForce -> M-site force redistribution -> SETTLE
velocities -> Nose-Hoover stepFinal.  Used as the timed CPU baseline of
bench.py (the reference has no CPU force path of its own) and by tests.
"""
from __future__ import annotations

import time

import numpy as np

from . import oracle as O

QQR = O.REAL_UNITS["qqr_to_eng"]


class SkinLists:
    """The neighbour list of the CPU step, kept between rebuilds by the
    reference's rule (GridGPU.cu:755-774 setBuildFlag with the
    periodicInterval gate of IntegratorVerlet.cu:696): at a turn that is a
    multiple of `interval`, rebuild iff some atom moved more than skin/2
    (minimum image) since the last build; the first call always builds."""

    def __init__(self, lo, L, rcut, skin, interval=10):
        self.lo, self.L = np.asarray(lo, np.float64), np.asarray(L, np.float64)
        self.cut = np.float32(float(np.float32(rcut)) + skin)
        self.skin, self.interval = skin, interval
        self.x_last = None
        self.lists = None
        self.builds = 0

    def get(self, x, turn, excl=None):
        if self.x_last is not None and (turn % self.interval != 0):
            return self.lists
        if self.x_last is not None:
            d = x - self.x_last
            d -= self.L * np.rint(d / self.L)
            if np.max(np.einsum("ij,ij->i", d, d)) <= 0.25 * self.skin * self.skin:
                return self.lists
        xs4 = np.zeros((len(x), 4), np.float32)
        xs4[:, :3] = x
        O.wrap_f32(xs4, self.lo, self.L)
        self.lists = O.nlist_cells(xs4, self.lo, self.L, self.cut, ids=np.arange(len(x)) if excl is not None else None,
                                   excl=excl)
        self.x_last = np.array(x, np.float64)
        self.builds += 1
        return self.lists

    def current(self, x, excl=None):
        """the list in force (built on first use)"""
        return self.lists if self.lists is not None else self.get(x, 0, excl=excl)


class WaterCPU:
    def __init__(self, sysd, e3b=False, rcut=9.0, skin=1.0, dt=2.0, grid=64, T=298.0, tau=100.0, interval=10):
        from md_engine_b200 import systems as S
        self.s = sysd
        self.e3b = e3b
        self.rcut, self.skin, self.dt, self.grid = rcut, skin, dt, grid
        self.x = np.asarray(sysd.pos, np.float64).copy()
        self.v = np.asarray(sysd.vel, np.float64).copy()
        self.m = sysd.mass
        self.invm = np.where(self.m > 0, 1.0 / np.where(self.m > 0, self.m, 1.0), 1e30)
        self.mol = sysd.molecules
        self.rd = O.RigidData("TIP4P/2005", S.MASS_O, S.MASS_H)
        bonds = []
        for o, h1, h2, mm in self.mol:
            bonds += [(o, h1), (o, h2), (h1, h2), (o, mm)]
        self.excl = O.exclusions_from_bonds(len(self.x), bonds)
        sig = {(0, 0): S.SIG_OO, (1, 1): 0.0, (0, 1): 0.0, (2, 2): 0.0}
        eps = {(0, 0): S.EPS_OO, (1, 1): 0.0, (0, 1): 0.0, (2, 2): 0.0}
        self.params = O.lj_params(3, sig, eps, rcut)
        self.alpha = O.p3m_alpha(sysd.q, len(self.x), sysd.L, (grid,) * 3, rcut)
        self.G = O.p3m_green(sysd.L, (grid,) * 3, self.alpha)
        self.ftm = O.REAL_UNITS["ftm_to_v"]
        self.turn = 0
        self.lists = SkinLists(sysd.lo, sysd.L, rcut, skin, interval)
        ndf = 6 * len(self.mol)
        self.nh = O.NoseHooverChain(T, tau, ndf, O.REAL_UNITS["boltz"], dt) if T is not None else None
        self.f = self.forces()  # forceInitial, before FixRigid::prepareForRun
        self.initial_constraints()
        if self.nh is not None:
            self.nh.prepare(O.kinetic_sum(self.v, self.invm) * O.REAL_UNITS["mvv_to_eng"])
        self.pending = 1.0

    def initial_constraints(self):
        """FixRigid::prepareForRun with solveInitialConstraints
        (FixRigid.cu:1740-1880): SETTLE onto itself, M sites, velocity
        constraints, centre-of-mass velocity removal over all atoms."""
        s, mol = self.s, self.mol
        x0 = self.x[mol[:, :3]].copy()
        xn, vn = O.settle_positions(x0, x0.copy(), self.v[mol[:, :3]], s.L, self.rd, self.dt)
        self.x[mol[:, :3]] = xn
        self.v[mol[:, :3]] = vn
        self.x[mol[:, 3]] = O.msite_positions(xn[:, 0], xn[:, 1], xn[:, 2], s.L, self.rd.r_OM)
        self.v[mol[:, :3]] = O.settle_velocities(self.x[mol[:, :3]], self.v[mol[:, :3]], s.L, self.rd)
        m = np.where(self.m > 0, self.m, 1e-30)
        vcom = np.sum(self.v * m[:, None], 0) / np.sum(m)
        self.v -= vcom

    def forces(self):
        s = self.s
        c, nb = self.lists.current(self.x, excl=self.excl)
        f = O.pair_forces(self.x, s.types, s.q, self.params, s.L, c, nb, qrc=self.rcut, alpha=self.alpha,
                          qqr_to_eng=QQR)["f"]
        f += O.p3m_forces(self.x, s.q, s.lo, s.L, (self.grid,) * 3, self.alpha, G=self.G)
        if self.e3b:
            f += O.e3b_forces(self.mol, self.x, s.L, O.e3b_params("E3B3"))[0]
        return f

    def step(self):
        s, mol, dt = self.s, self.mol, self.dt
        dtf = 0.5 * dt * self.ftm
        # the turn's list check comes first (IntegratorVerlet.cu:696-698)
        self.lists.get(self.x, self.turn, excl=self.excl)
        if self.nh is not None:
            self.pending *= self.nh.integrate(True)
            self.v *= self.pending
        real = self.m > 0
        x0 = self.x[mol[:, :3]].copy()
        self.v[real] += dtf * self.f[real] * self.invm[real][:, None]
        self.v[~real] = 0.0
        self.x[real] += dt * self.v[real]
        xn, vn = O.settle_positions(x0, self.x[mol[:, :3]], self.v[mol[:, :3]], s.L, self.rd, dt)
        self.x[mol[:, :3]] = xn
        self.v[mol[:, :3]] = vn
        self.x[mol[:, 3]] = O.msite_positions(xn[:, 0], xn[:, 1], xn[:, 2], s.L, self.rd.r_OM)
        self.f = self.forces()
        self.v[real] += dtf * self.f[real] * self.invm[real][:, None]
        fO, fH1, fH2, vO, vH1, vH2 = O.msite_distribute(
            self.f[mol[:, 0]], self.f[mol[:, 1]], self.f[mol[:, 2]], self.f[mol[:, 3]],
            self.v[mol[:, 0]], self.v[mol[:, 1]], self.v[mol[:, 2]], 1.0 / self.rd.mO, 1.0 / self.rd.mH,
            self.rd.gamma, dtf)
        self.f[mol[:, 0]], self.f[mol[:, 1]], self.f[mol[:, 2]] = fO, fH1, fH2
        self.f[mol[:, 3]] = 0.0
        self.v[mol[:, 0]], self.v[mol[:, 1]], self.v[mol[:, 2]] = vO, vH1, vH2
        self.v[mol[:, :3]] = O.settle_velocities(self.x[mol[:, :3]], self.v[mol[:, :3]], s.L, self.rd)
        if self.nh is not None:
            self.nh.ke = O.kinetic_sum(self.v, self.invm) * O.REAL_UNITS["mvv_to_eng"]
            self.pending = self.nh.integrate(False)
        self.turn += 1

    def end_of_run(self):
        """FixNoseHoover::postRun applies the scale left by the last stepFinal"""
        self.v *= self.pending
        self.pending = 1.0


class LJCPU:
    def __init__(self, sysd, rcut=2.5, skin=0.3, dt=0.005, T=1.2, tau=0.5, interval=10):
        self.s = sysd
        self.rcut, self.skin, self.dt = rcut, skin, dt
        self.x = np.asarray(sysd.pos, np.float64).copy()
        self.v = np.asarray(sysd.vel, np.float64).copy()
        self.m = sysd.mass
        self.params = O.lj_params(1, {(0, 0): 1.0}, {(0, 0): 1.0}, rcut)
        self.turn = 0
        self.lists = SkinLists(sysd.lo, sysd.L, rcut, skin, interval)
        self.nh = O.NoseHooverChain(T, tau, 3 * len(self.x), 1.0, dt)
        self.f = self.forces()
        self.nh.prepare(float(np.sum(self.m[:, None] * self.v ** 2)))
        self.pending = 1.0

    def forces(self):
        s = self.s
        c, nb = self.lists.current(self.x)
        return O.pair_forces(self.x, s.types, None, self.params, s.L, c, nb)["f"]

    def step(self):
        dtf = 0.5 * self.dt
        self.lists.get(self.x, self.turn)
        self.pending *= self.nh.integrate(True)
        self.v *= self.pending
        self.v += dtf * self.f / self.m[:, None]
        self.x += self.dt * self.v
        self.f = self.forces()
        self.v += dtf * self.f / self.m[:, None]
        self.nh.ke = float(np.sum(self.m[:, None] * self.v ** 2))
        self.pending = self.nh.integrate(False)
        self.turn += 1


def water_reference(sysd, x, rcut=9.0, skin=1.0, grid=64, alpha=None, e3b=False):
    """FP64 per-site forces (pair + P3M reciprocal [+ E3B]), energies per term
    and the total virial of a rigid-water configuration x, with the list of
    the same FP32 predicate and exclusions; alpha as the library's (or the
    reference secant when None)."""
    from md_engine_b200 import systems as S
    bonds = []
    for o, h1, h2, mm in sysd.molecules:
        bonds += [(o, h1), (o, h2), (h1, h2), (o, mm)]
    excl = O.exclusions_from_bonds(len(x), bonds)
    sig = {(0, 0): S.SIG_OO, (1, 1): 0.0, (0, 1): 0.0, (2, 2): 0.0}
    eps = {(0, 0): S.EPS_OO, (1, 1): 0.0, (0, 1): 0.0, (2, 2): 0.0}
    params = O.lj_params(3, sig, eps, rcut)
    if alpha is None:
        alpha = O.p3m_alpha(sysd.q, len(x), sysd.L, (grid,) * 3, rcut)
    xs4 = np.zeros((len(x), 4), np.float32)
    xs4[:, :3] = x
    O.wrap_f32(xs4, sysd.lo, sysd.L)
    cut = np.float32(float(np.float32(rcut)) + skin)
    c, nb = O.nlist_cells(xs4, sysd.lo, sysd.L, cut, ids=np.arange(len(x)), excl=excl)
    pr = O.pair_forces(x, sysd.types, sysd.q, params, sysd.L, c, nb, qrc=rcut, alpha=alpha, qqr_to_eng=QQR,
                       want=("f", "virial", "energy"))
    vir = pr["virial"].sum(0)
    frec, erec = O.p3m_forces(x, sysd.q, sysd.lo, sysd.L, (grid,) * 3, alpha, want_energy=True, virial=vir)
    q2 = QQR * float(np.sum(np.asarray(sysd.q, np.float64) ** 2))
    f = pr["f"] + frec
    energy = {"pair": float(pr["energy"].sum()), "p3m": float(erec - alpha / np.sqrt(np.pi) * q2)}
    if e3b:
        fe, (e2, e3), _ = O.e3b_forces(sysd.molecules, x, sysd.L, O.e3b_params("E3B3"), virial=vir)
        f = f + fe
        energy["e3b2"], energy["e3b3"] = float(e2), float(e3)
    return {"f": f, "energy": energy, "virial": vir}


def lj_reference(sysd, x, rcut=2.5, skin=0.3):
    """FP64 LJ forces, energy and total virial of configuration x"""
    params = O.lj_params(1, {(0, 0): 1.0}, {(0, 0): 1.0}, rcut)
    xs4 = np.zeros((len(x), 4), np.float32)
    xs4[:, :3] = x
    O.wrap_f32(xs4, sysd.lo, sysd.L)
    cut = np.float32(float(np.float32(rcut)) + skin)
    c, nb = O.nlist_cells(xs4, sysd.lo, sysd.L, cut)
    pr = O.pair_forces(x, sysd.types, None, params, sysd.L, c, nb, want=("f", "virial", "energy"))
    return {"f": pr["f"], "energy": {"pair": float(pr["energy"].sum())}, "virial": pr["virial"].sum(0)}


def time_steps(sysd, name, nsample=1, warmup=0, repeats=1):
    """Time the named workload's whole CPU step: `warmup` untimed steps, then
    `repeats` samples of `nsample` consecutive steps each; the neighbour list
    is kept between checks by the reference's skin rule (every 10 steps).
    steps_per_s is the median over the samples."""
    if name == "lj":
        sim = LJCPU(sysd)
        desc = f"{len(sysd.pos)}-atom LJ"
    else:
        sim = WaterCPU(sysd, e3b=(name == "water_e3b"))
        desc = f"{len(sysd.molecules)}-molecule TIP4P/2005" + ("+E3B3" if name == "water_e3b" else "")
    for _ in range(warmup):
        sim.step()
    rates = []
    b0 = sim.lists.builds
    for _ in range(max(1, repeats)):
        t0 = time.perf_counter()
        for _ in range(nsample):
            sim.step()
        rates.append(nsample / (time.perf_counter() - t0))
    builds = sim.lists.builds - b0
    total = nsample * max(1, repeats)
    return {"steps_per_s": float(np.median(rates)), "cores": O.num_threads(), "samples": rates,
            "list_builds": builds,
            "sample": f"median of {max(1, repeats)} x {nsample} consecutive FP64 timesteps of the {desc} system "
                      f"after {warmup} warm-up (oracle port: OpenMP pair/nlist, numpy P3M/SETTLE; neighbour list "
                      f"rebuilt by the skin rule every 10 steps: {builds} builds in {total} steps)",
            "workload": desc, "sim": sim}
