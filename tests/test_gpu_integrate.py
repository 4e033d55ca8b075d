"""Integrator, SETTLE and Nose-Hoover stages vs the oracle, plus whole-step
consistency (fused CUDA-graph step vs the reference's hook-by-hook order)
and NVE energy drift."""
import numpy as np
import pytest

from md_engine_b200 import Bounds, FixLJCut, IntegratorVerlet, State, Vector, systems
from tests.helpers import water_small

pytestmark = pytest.mark.gpu


def test_free_particle_verlet():
    """tests/Integrators/test_IntegratorVerlet.py:62-132: a free particle with
    velocity 1 moves dt*N*v (FP32 positions: tolerance is FP32 rounding)."""
    st = State()
    st.units.setLJ()
    st.bounds = Bounds(st, lo=Vector(0, 0, 0), hi=Vector(100, 100, 100))
    st.rCut = 9.0
    st.padding = 1.0
    st.periodicInterval = 1
    st.dt = 0.005
    st.atomParams.addSpecies("test", 1.0, 1)
    st.addAtom("test", Vector(20.0, 20.0, 20.0))
    lj = FixLJCut(st, "lj")
    lj.setParameter("sig", "test", "test", 1.0)
    lj.setParameter("eps", "test", "test", 1.0)
    st.activateFix(lj)
    st.setVelocities([0], [[1.0, 0.0, 0.0]])
    IntegratorVerlet(st).run(10000)
    x, v, _ = st.getAtoms()
    # FP32 positions: x += 0.005 rounds by a near-constant fraction of an ulp
    # each step (the reference test notes it only passes in double precision)
    assert abs(x[0, 0] - (20.0 + 0.005 * 10000)) < 2e-2
    assert x[0, 1] == 20.0 and x[0, 2] == 20.0
    assert v[0, 0] == 1.0


def _rigid_positions(st, mol):
    x, v, f = st.getAtoms()
    return x[mol[:, :3]], v[mol[:, :3]], x, v, f


def test_settle_positions_and_velocities_vs_oracle(oracle):
    sysd = water_small(seed=21)
    st, fx = systems.build_water_state(sysd, rcut=6.5, skin=1.0, grid=32, alpha=0.35, thermostat=False)
    st.prepare()
    rigid = fx["rigid"]
    mol = sysd.molecules
    rd = oracle.RigidData("TIP4P/2005", systems.MASS_O, systems.MASS_H)
    # save_prev then an unconstrained drift of the real atoms
    rigid.savePrev()
    x0m, v0m, x, v, _ = _rigid_positions(st, mol)
    rng = np.random.default_rng(1)
    dt = 2.0
    xn = x.copy()
    kick = rng.normal(0, 0.01, (len(x), 3))
    kick[mol[:, 3]] = 0.0
    xn += kick
    st.putAtoms(positions=xn)
    rigid.settlePositions()
    xs, vs, xg, vg, _ = _rigid_positions(st, mol)
    xo, vo = oracle.settle_positions(x0m, np.asarray(xn[mol[:, :3]], np.float32).astype(np.float64),
                                     np.asarray(v[mol[:, :3]], np.float32).astype(np.float64), sysd.L, rd, dt)
    assert np.max(np.abs(xs - xo)) < 2e-5
    assert np.max(np.abs(vs - vo)) < 1e-5 * max(1.0, np.abs(vo).max())
    # bond lengths restored
    dOH = np.linalg.norm(xs[:, 1] - xs[:, 0], axis=1)
    assert np.max(np.abs(dOH - rd.r_OH)) < 2e-5
    # M site placed from the constrained triangle
    m = oracle.msite_positions(xg[mol[:, 0]], xg[mol[:, 1]], xg[mol[:, 2]], sysd.L, rd.r_OM)
    assert np.max(np.abs(xg[mol[:, 3]] - m)) < 2e-5
    # velocity constraint
    vin = vg.copy()
    vin[mol[:, :3]] += rng.normal(0, 0.005, vin[mol[:, :3]].shape)
    st.putAtoms(velocities=vin)
    rigid.settleVelocities()
    _, _, xg, vg2, _ = _rigid_positions(st, mol)
    vref = oracle.settle_velocities(xg[mol[:, :3]], np.asarray(vin[mol[:, :3]], np.float32).astype(np.float64),
                                    sysd.L, rd)
    assert np.max(np.abs(vg2[mol[:, :3]] - vref)) < 1e-6 * max(1.0, np.abs(vref).max()) + 1e-7
    # relative velocity along every bond is zero afterwards
    for a, b in ((0, 1), (0, 2), (1, 2)):
        d = xg[mol[:, a]] - xg[mol[:, b]]
        rel = np.sum((vg2[mol[:, a]] - vg2[mol[:, b]]) * d, 1)
        assert np.max(np.abs(rel)) < 1e-5


def _total_energy(st):
    ke2, _ = st.kinetic()
    return 0.5 * ke2 + float(np.sum(st.potentialEnergy()))


def test_lj_nve_energy_drift():
    sysd = systems.lj_fcc(ncell=8, seed=3)
    st, _ = systems.build_lj_state(sysd, rcut=2.5, skin=0.3, dt=0.005, interval=10)
    it = IntegratorVerlet(st)
    it.run(10)
    e0 = _total_energy(st)
    it.run(1000)
    e1 = _total_energy(st)
    n = len(sysd.pos)
    # per-atom drift over 1000 steps of 0.005 tau: shifted-energy LJ, FP32
    assert abs(e1 - e0) / n < 5e-3, (e0, e1)


def test_fused_step_matches_hook_by_hook():
    """the CUDA-graph fused timestep and the one-kernel-per-reference-hook
    order give the same trajectory to FP32 rounding over 20 water steps"""
    out = []
    for mode in (0, 1):
        sysd = water_small(seed=2)
        st, _ = systems.build_water_state(sysd, rcut=6.5, skin=1.0, grid=32, e3b=True, alpha=0.35,
                                          thermostat=True, interval=5)
        it = IntegratorVerlet(st)
        it.setMode(mode)
        it.run(20)
        x, v, f = st.getAtoms()
        out.append((x, v))
    dx = np.max(np.abs(out[0][0] - out[1][0]))
    dv = np.max(np.abs(out[0][1] - out[1][1]))
    assert dx < 1e-3 and dv < 1e-3, (dx, dv)


def _oracle_lj_run(O, sysd, nsteps, dt, T, tau, rcut=2.5, skin=0.3):
    """reference step order (IntegratorVerlet.cu:694-754) in FP64 with the
    oracle's pair forces and Nose-Hoover chain"""
    x = np.asarray(sysd.pos, np.float32).astype(np.float64)
    v = np.asarray(sysd.vel, np.float32).astype(np.float64)
    m = sysd.mass
    params = O.lj_params(1, {(0, 0): 1.0}, {(0, 0): 1.0}, rcut)
    cut = np.float32(float(np.float32(rcut)) + skin)

    def forces(x):
        xs4 = np.zeros((len(x), 4), np.float32)
        xs4[:, :3] = x
        xs4 = O.wrap_f32(xs4, sysd.lo, sysd.L)
        c, nb = O.nlist_cells(xs4, sysd.lo, sysd.L, cut)
        return O.pair_forces(x, sysd.types, None, params, sysd.L, c, nb)["f"]

    f = forces(x)
    nh = O.NoseHooverChain(T, tau, 3 * len(x), 1.0, dt)
    nh.prepare(float(np.sum(m[:, None] * v * v)))
    pending = 1.0
    dtf = 0.5 * dt
    for _ in range(nsteps):
        pending *= nh.integrate(True)
        v *= pending
        v += dtf * f / m[:, None]
        x += dt * v
        f = forces(x)
        v += dtf * f / m[:, None]
        nh.ke = float(np.sum(m[:, None] * v * v))
        pending = nh.integrate(False)
    return x, v * pending


def test_lj_nvt_trajectory_vs_oracle(oracle):
    """20 NVT steps of an 864-atom LJ fluid: the device Nose-Hoover chain,
    Verlet halves and pair forces track the FP64 oracle step by step"""
    sysd = systems.lj_fcc(ncell=6, seed=9)
    st, _ = systems.build_lj_state(sysd, rcut=2.5, skin=0.3, dt=0.005, T=1.5, tau=0.5, interval=1)
    IntegratorVerlet(st).run(20)
    x, v, _ = st.getAtoms()
    xo, vo = _oracle_lj_run(oracle, sysd, 20, 0.005, 1.5, 0.5)
    d = x - xo
    d -= sysd.L * np.rint(d / sysd.L)
    assert np.max(np.abs(d)) < 1e-4
    # both apply the last stepFinal scale at the end of the run (postRun)
    assert np.max(np.abs(v - vo)) < 1e-3 * np.abs(vo).max()


def test_water_nvt_runs_and_holds_constraints():
    sysd = water_small(seed=4)
    st, _ = systems.build_water_state(sysd, rcut=6.5, skin=1.0, grid=32, e3b=True, T=298.0, tau=100.0, interval=10)
    it = IntegratorVerlet(st)
    it.run(200)
    x, v, f = st.getAtoms()
    mol = sysd.molecules
    L = sysd.L
    for a, b, ref in ((0, 1, 0.9572), (0, 2, 0.9572), (1, 2, 1.5139)):
        d = x[mol[:, a]] - x[mol[:, b]]
        d -= L * np.rint(d / L)
        assert np.max(np.abs(np.linalg.norm(d, axis=1) - ref)) < 1e-4
    bits, maxn, nb = st.status()
    assert bits == 0
    mv2, ndf = st.kinetic()
    T = mv2 * systems.MVV_TO_ENG_REAL / (ndf * systems.BOLTZ_REAL)
    # a random-orientation lattice releases potential energy for ~1 ps
    assert 150 < T < 1200


@pytest.mark.parametrize("e3b", [False, True])
def test_water_trajectory_vs_oracle(oracle, e3b):
    """10 NVT steps of rigid TIP4P/2005 (+E3B3): the fused CUDA-graph step
    against the whole-step FP64 oracle in the reference hook order
    (oracle/cpu_step.py), from the same seeded start"""
    from oracle.cpu_step import WaterCPU
    sysd = water_small(seed=12)
    st, fx = systems.build_water_state(sysd, rcut=6.5, skin=1.0, grid=32, e3b=e3b, T=298.0, tau=100.0, interval=10)
    IntegratorVerlet(st).run(10)
    x, v, _ = st.getAtoms()
    sim = WaterCPU(sysd, e3b=e3b, rcut=6.5, skin=1.0, dt=2.0, grid=32, T=298.0, tau=100.0)
    assert abs(sim.alpha - fx["ewald"].alpha) < 1e-9
    for _ in range(10):
        sim.step()
    sim.end_of_run()
    d = x - sim.x
    d -= sysd.L * np.rint(d / sysd.L)
    assert np.max(np.abs(d)) < 1e-3, np.max(np.abs(d))
    real = sysd.mass > 0
    assert np.max(np.abs(v[real] - sim.v[real])) < 1e-3 * np.abs(sim.v[real]).max()


def test_water_nve_energy_conservation():
    """rigid TIP4P/2005 NVE, 1 fs: total energy drift stays small (FP32 forces,
    FP64 SETTLE); reported per molecule"""
    sysd = water_small(seed=6)
    st, _ = systems.build_water_state(sysd, rcut=6.5, skin=1.0, grid=32, dt=1.0, thermostat=False, interval=10)
    it = IntegratorVerlet(st)
    it.run(200)  # let the lattice relax a little
    e0 = _total_energy_real(st)
    it.run(500)
    e1 = _total_energy_real(st)
    drift = abs(e1 - e0) / len(sysd.molecules)
    assert drift < 0.05, (e0, e1, drift)


def _total_energy_real(st):
    mv2, _ = st.kinetic()
    return 0.5 * mv2 * systems.MVV_TO_ENG_REAL + float(np.sum(st.potentialEnergy()))


def test_autotune_keeps_the_state_and_the_trajectory():
    """IntegratorVerlet.autotune (Integrator::tune's role): the molecule
    form's pair grid cap is timed on the force phase alone; positions,
    velocities and forces are left as they were, the chosen cap is kept on
    the state, and the run that follows equals the same run without the
    tuning (the grid shape changes no force; to the float-atomic order of
    the P3M spread)"""
    from md_engine_b200 import IntegratorVerlet
    sysd = systems.water_tip4p2005(nside=10, seed=5)
    a, _ = systems.build_water_state(sysd, rcut=9.0, skin=1.0, grid=32)
    b, _ = systems.build_water_state(sysd, rcut=9.0, skin=1.0, grid=32)
    ia, ib = IntegratorVerlet(a), IntegratorVerlet(b)
    ia.run(5)
    ib.run(5)
    x0, v0, f0 = a.getAtoms()
    cap, ms = ia.autotune(reps=4, caps=(4, 10, -1))
    assert cap in (4, 10, -1) and ms > 0
    assert int(a.pairBlocksPerSM) == cap
    x1, v1, f1 = a.getAtoms()
    assert np.array_equal(x0, x1) and np.array_equal(v0, v1) and np.array_equal(f0, f1)
    ia.run(20)
    ib.run(20)
    xa, _, _ = a.getAtoms()
    xb, _, _ = b.getAtoms()
    d = xa - xb
    d -= sysd.L * np.rint(d / sysd.L)
    assert np.abs(d).max() < 1e-3
    # the per-site form has no such shape
    lj = systems.lj_fcc(ncell=6, seed=3)
    st, _ = systems.build_lj_state(lj, rcut=2.5, skin=0.3)
    assert IntegratorVerlet(st).autotune(reps=2) == (0, 0.0)
