"""FP64 restatement of FixNoseHoover's isotropic MTK barostat -- TEST
INFRASTRUCTURE ONLY (nothing in the package imports it).

One NPT step of an LJ fluid in the reference's hook order
(IntegratorVerlet.cu:694-754 with requiresPostNVE_V) and FixNoseHoover's
propagator (FixNoseHoover.cu: stepInit :413-518, postNVE_V :520-536,
stepFinal :544-605, updateBarostatMasses :628-667,
updateBarostatThermalMasses :669-700, barostatThermostatIntegrate :702-793,
barostatVelocityIntegrate :868-943, scaleVelocitiesBarostat :945-1015,
rescaleVolume :1017-1032; Mod::scaleSystem about the box centre, Mod.cu:
201-240), LJ units (boltz = mvv_to_eng = nktv_to_press = ftm_to_v = 1).
Forces, virials and the cell list are the oracle's (oracle.py), on a list
rebuilt every step (the box moves every step).

Parity: the barostat propagators (masses, thermal masses, the barostat
chain, the cell-velocity kick) are pinned against the reference's own
FixNoseHoover.cu compiled from source on the CPU (oracle/ref_nh_harness.cu
-> oracle/_ref/librefbarostat.so; fixture tests/golden/ref_barostat.json): with
barostat_velocity(ref_float=True) and a float time step this restatement
reproduces the reference bit for bit; in FP64 (the library's precision) it
differs only by the reference's float rounding of the pressure, the cell
kick, the volume and the time step.  The step's hook order, the particle
scaling factors and the volume rescale remain a restatement checked against
the library's MTK step (their kernels and the pressure computer are not run
by the harness), and, for the physics, by an LJ fluid reaching its set
pressure at the density this propagator gives."""
from __future__ import annotations

import math

import numpy as np

from . import oracle as O


class MTKLJ:
    def __init__(self, sysd, T, tau, P, ptau, rcut=2.5, skin=0.3, dt=0.005, chain=10):
        self.s = sysd
        self.rcut, self.skin, self.dt = rcut, skin, dt
        self.x = np.asarray(sysd.pos, np.float64).copy()
        self.v = np.asarray(sysd.vel, np.float64).copy()
        self.m = np.asarray(sysd.mass, np.float64)
        self.lo = np.asarray(sysd.lo, np.float64).copy()
        self.L = np.asarray(sysd.L, np.float64).copy()
        self.params = O.lj_params(1, {(0, 0): 1.0}, {(0, 0): 1.0}, rcut)
        self.n = len(self.x)
        self.ndf = 3 * self.n
        self.T, self.P, self.pfreq = T, P, 1.0 / ptau
        self.nh = O.NoseHooverChain(T, tau, self.ndf, 1.0, dt, chain)
        self.pc = chain
        self.pvel = [0.0, 0.0, 0.0]
        self.pmass = [0.0, 0.0, 0.0]
        self.ptv = [0.0] * chain
        self.ptf = [0.0] * chain
        self.ptm = [0.0] * chain
        self.pending = 1.0
        self.f, self.w = self.forces()
        self.nh.prepare(self.kinetic())
        self.barostat_masses()
        self.barostat_thermal_masses()
        self.last_pressure = None

    # -- forces and observables ------------------------------------------
    def forces(self):
        xs4 = np.zeros((self.n, 4), np.float32)
        xs4[:, :3] = self.x
        O.wrap_f32(xs4, self.lo, self.L)
        cut = np.float32(float(np.float32(self.rcut)) + self.skin)
        c, nb = O.nlist_cells(xs4, self.lo, self.L, cut)
        pr = O.pair_forces(self.x, self.s.types, None, self.params, self.L, c, nb, want=("f", "virial"))
        return pr["f"], pr["virial"].sum(0)

    def kinetic(self):
        return float(np.sum(self.m[:, None] * self.v ** 2))

    def volume(self):
        return float(np.prod(self.L))

    def pressure(self, ke):
        return (ke + self.w[0] + self.w[1] + self.w[2]) / (3.0 * self.volume())

    # -- barostat pieces ---------------------------------------------------
    def barostat_masses(self):
        kt = self.T
        for i in range(3):
            self.pmass[i] = (self.ndf + 3.0) * kt / (self.pfreq * self.pfreq)

    def barostat_thermal_masses(self):
        kt = self.T
        self.ptm[0] = 3.0 * 4.0 * kt / (2.0 * self.pfreq)
        for i in range(1, self.pc):
            self.ptm[i] = kt / (self.pfreq * self.pfreq)
        for i in range(1, self.pc):
            self.ptf[i] = (self.ptm[i - 1] * self.ptv[i - 1] * self.ptv[i - 1] - kt) / self.ptm[i]

    def ke_barostat(self):
        ke = 0.0
        for i in range(3):
            ke += self.pmass[i] * self.pvel[i] * self.pvel[i]
        return ke

    def barostat_thermostat(self, step_init):
        kt, n = self.T, self.pc
        v, F, M = self.ptv, self.ptf, self.ptm
        if not step_init:
            F[0] = (self.ke_barostat() - kt) / M[0]
        ts = self.dt
        t2, t4, t8 = 0.5 * ts, 0.25 * ts, 0.125 * ts
        v[n - 1] += t4 * F[n - 1]
        for k in range(n - 2, 0, -1):
            pf = math.exp(-t8 * v[k + 1])
            v[k] = (v[k] * pf + t4 * F[k]) * pf
        pf = math.exp(-t8 * v[1])
        v[0] = (v[0] * pf + t4 * F[0]) * pf
        sc = math.exp(-t2 * v[0])
        self.pvel = [p * sc for p in self.pvel]
        v[0] *= pf
        F[0] = (self.ke_barostat() - kt) / M[0]
        v[0] += t4 * F[0]
        v[0] *= pf
        for k in range(1, n - 1):
            pf = math.exp(-t8 * v[k + 1])
            v[k] *= pf
            F[k] = (M[k - 1] * v[k - 1] * v[k - 1] - kt) / M[k]
            v[k] += t4 * F[k]
            v[k] *= pf
        F[n - 1] = (M[n - 2] * v[n - 2] * v[n - 2] - kt) / M[n - 1]
        v[n - 1] += t4 * F[n - 1]

    def barostat_velocity(self, ke, p, ref_float=False):
        """the cell-velocity kick in FP64; with ref_float, in the reference's
        own precision: its pressure tensor and the kick G are Virials of
        floats (Virial.h:10), the volume the float product of the float box
        lengths (BoundsGPU.h:110-112), the time step a float (State.h:117)"""
        tcur = ke / self.ndf
        alpha = tcur * self.ndf / (self.n * 3.0)
        if ref_float:
            f32 = np.float32
            V = float(f32(f32(self.L[0]) * f32(self.L[1])) * f32(self.L[2]))
            pf, dt = float(f32(p)), f32(self.dt)
            for i in range(3):
                G = f32(alpha / self.pmass[i])
                G = f32(float(G) + (pf - self.P) * V / self.pmass[i])
                self.pvel[i] += float(G * dt) * 0.5
            return
        for i in range(3):
            G = alpha / self.pmass[i] + (p - self.P) * self.volume() / self.pmass[i]
            self.pvel[i] += G * self.dt * 0.5

    def scale_velocities(self):
        alpha = sum(self.pvel) / (3.0 * self.n)
        x = (self.pvel[0] + alpha) * self.dt * 0.25
        x2 = x * x
        x4 = x2 * x2
        add = x2 / 6.0 + x4 / 120.0 + x4 * x2 / 5040.0 + x4 * x4 / 362880.0
        mult = math.exp(-x)
        dtf = 0.5 * self.dt
        self.v = (self.v * mult + dtf * self.f / self.m[:, None] * add) * mult

    def rescale_volume(self):
        sc = math.exp(self.pvel[0] * self.dt)
        c = self.lo + 0.5 * self.L
        self.x = c + (self.x - c) * sc
        self.L = self.L * sc
        self.lo = c - 0.5 * self.L

    def restart(self):
        """the end of one run and the start of the next: postRun applies
        the pending thermostat scale (FixNoseHoover.cu:406-411), prepareFinal
        recomputes the particle chain's forces and restarts the barostat
        variables at rest (FixNoseHoover.cu:240-404)"""
        self.v *= self.pending
        self.pending = 1.0
        self.nh.prepare(self.kinetic())
        self.pvel = [0.0, 0.0, 0.0]
        self.pmass = [0.0, 0.0, 0.0]
        self.ptv = [0.0] * self.pc
        self.ptf = [0.0] * self.pc
        self.ptm = [0.0] * self.pc
        self.barostat_masses()
        self.barostat_thermal_masses()

    # -- one step ------------------------------------------------------------
    def step(self):
        dtf = 0.5 * self.dt
        self.barostat_masses()
        self.barostat_thermal_masses()
        self.barostat_thermostat(True)
        self.pending *= self.nh.integrate(True)
        self.v *= self.pending
        self.pending = 1.0
        ke = self.kinetic()
        self.barostat_velocity(ke, self.pressure(ke))
        self.v += dtf * self.f / self.m[:, None]
        self.scale_velocities()
        self.rescale_volume()
        self.x += self.dt * self.v
        self.f, self.w = self.forces()
        self.v += dtf * self.f / self.m[:, None]
        self.scale_velocities()
        ke = self.kinetic()
        p = self.pressure(ke)
        self.last_pressure = p
        self.barostat_velocity(ke, p)
        self.nh.ke = ke
        self.pending *= self.nh.integrate(False)
        self.barostat_masses()
        self.barostat_thermal_masses()
        self.barostat_thermostat(False)
