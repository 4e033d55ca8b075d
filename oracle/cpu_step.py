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


class WaterCPU:
    def __init__(self, sysd, e3b=False, rcut=9.0, skin=1.0, dt=2.0, grid=64, T=298.0, tau=100.0):
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
        xs4 = np.zeros((len(self.x), 4), np.float32)
        xs4[:, :3] = self.x
        O.wrap_f32(xs4, s.lo, s.L)
        cut = np.float32(float(np.float32(self.rcut)) + self.skin)
        c, nb = O.nlist_cells(xs4, s.lo, s.L, cut, ids=np.arange(len(self.x)), excl=self.excl)
        f = O.pair_forces(self.x, s.types, s.q, self.params, s.L, c, nb, qrc=self.rcut, alpha=self.alpha,
                          qqr_to_eng=QQR)["f"]
        f += O.p3m_forces(self.x, s.q, s.lo, s.L, (self.grid,) * 3, self.alpha, G=self.G)
        if self.e3b:
            f += O.e3b_forces(self.mol, self.x, s.L, O.e3b_params("E3B3"))[0]
        return f

    def step(self):
        s, mol, dt = self.s, self.mol, self.dt
        dtf = 0.5 * dt * self.ftm
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

    def end_of_run(self):
        """FixNoseHoover::postRun applies the scale left by the last stepFinal"""
        self.v *= self.pending
        self.pending = 1.0


class LJCPU:
    def __init__(self, sysd, rcut=2.5, skin=0.3, dt=0.005, T=1.2, tau=0.5):
        self.s = sysd
        self.rcut, self.skin, self.dt = rcut, skin, dt
        self.x = np.asarray(sysd.pos, np.float64).copy()
        self.v = np.asarray(sysd.vel, np.float64).copy()
        self.m = sysd.mass
        self.params = O.lj_params(1, {(0, 0): 1.0}, {(0, 0): 1.0}, rcut)
        self.nh = O.NoseHooverChain(T, tau, 3 * len(self.x), 1.0, dt)
        self.f = self.forces()
        self.nh.prepare(float(np.sum(self.m[:, None] * self.v ** 2)))
        self.pending = 1.0

    def forces(self):
        s = self.s
        xs4 = np.zeros((len(self.x), 4), np.float32)
        xs4[:, :3] = self.x
        O.wrap_f32(xs4, s.lo, s.L)
        cut = np.float32(float(np.float32(self.rcut)) + self.skin)
        c, nb = O.nlist_cells(xs4, s.lo, s.L, cut)
        return O.pair_forces(self.x, s.types, None, self.params, s.L, c, nb)["f"]

    def step(self):
        dtf = 0.5 * self.dt
        self.pending *= self.nh.integrate(True)
        self.v *= self.pending
        self.v += dtf * self.f / self.m[:, None]
        self.x += self.dt * self.v
        self.f = self.forces()
        self.v += dtf * self.f / self.m[:, None]
        self.nh.ke = float(np.sum(self.m[:, None] * self.v ** 2))
        self.pending = self.nh.integrate(False)


def time_steps(sysd, name, nsample=1, warmup=0):
    """Time `nsample` whole CPU steps (after `warmup`) of the named workload."""
    if name == "lj":
        sim = LJCPU(sysd)
        desc = f"{len(sysd.pos)}-atom LJ"
    else:
        sim = WaterCPU(sysd, e3b=(name == "water_e3b"))
        desc = f"{len(sysd.molecules)}-molecule TIP4P/2005" + ("+E3B3" if name == "water_e3b" else "")
    for _ in range(warmup):
        sim.step()
    t0 = time.perf_counter()
    for _ in range(nsample):
        sim.step()
    dt = time.perf_counter() - t0
    return {"steps_per_s": nsample / dt, "cores": O.num_threads(),
            "sample": f"{nsample} full FP64 timestep(s) of the {desc} system (oracle port, OpenMP pair/nlist, "
                      f"numpy P3M/SETTLE), {warmup} warm-up",
            "workload": desc}
