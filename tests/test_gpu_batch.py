"""Batched replicas: independent water boxes of different sizes and
temperatures advanced by one launch per phase must follow the same
trajectories as the same boxes run one at a time through IntegratorVerlet
(same arithmetic per replica; only the float-atomic order of the P3M spread
and the batched FFT plans differ, so positions agree to well below 1e-3 A
after a few dozen steps)."""
import numpy as np
import pytest

from md_engine_b200 import BatchReplicas, IntegratorVerlet, kernel_launches, systems

pytestmark = pytest.mark.gpu

RCUT, SKIN = 9.0, 0.8


def _replica(nmol, T, seed, e3b=False):
    sysd = systems.water_tip4p2005(nmol=nmol, T=T, seed=seed)
    mesh = systems.p3m_mesh_for(sysd.L[0])
    st, fixes = systems.build_water_state(sysd, rcut=RCUT, skin=SKIN, grid=mesh, T=T, e3b=e3b)
    st.nThreadPerAtom = 8
    return st, fixes


def _trajectories(spec, nsteps, e3b=False, form=0):
    batch_states = [_replica(m, T, seed, e3b)[0] for m, T, seed in spec]
    if form:
        for st in batch_states:
            st.pairForm = form
    b = BatchReplicas(batch_states)
    b.prepare()
    forms = [int(st.pairForm) for st in batch_states]
    if form == 1:
        assert forms == [1] * len(spec)
    else:
        # each replica in its own form: the molecule form where its box holds
        # the molecule list's minimum image, the per-site form below that
        assert 1 in forms and 2 in forms, forms
    b.run(nsteps)
    xb = [st.getAtoms()[0] for st in batch_states]
    singles = []
    for m, T, seed in spec:
        st, _ = _replica(m, T, seed, e3b)
        IntegratorVerlet(st).run(nsteps)
        singles.append(st.getAtoms()[0])
    return xb, singles, batch_states


@pytest.mark.parametrize("form", [0, 1])
@pytest.mark.parametrize("e3b", [False, True])
def test_batch_matches_single_runs(e3b, form):
    # form 0: a mixed batch (the 256-molecule box too small for the molecule
    # form, the others in it); form 1: every replica per-site
    spec = [(256, 265.0, 11), (520, 300.0, 12), (700, 350.0, 13)] if form == 0 else \
        [(256, 265.0, 11), (311, 300.0, 12), (420, 350.0, 13)]
    xb, xs, states = _trajectories(spec, 25, e3b=e3b, form=form)
    for (m, T, seed), a, b in zip(spec, xb, xs):
        assert a.shape == (4 * m, 3)
        # positions compared by minimum image (in the per-site form the
        # batch stores periodic images of some sites differently from the
        # single run's molecule form between rebuilds)
        L = systems.water_tip4p2005(nmol=m, T=T, seed=seed).L
        d = a - b
        d -= L * np.rint(d / L)
        d = np.abs(d).max()
        assert d < 1e-3, f"replica of {m} molecules drifted {d} A from its single run"
    for st in states:
        assert st.status()[0] == 0


def _launches_per_step(b):
    """kernel launches per step (the per-call end-of-run work cancels out)"""
    b.run(10)  # captures the graphs
    k0 = kernel_launches()
    b.run(20)
    k1 = kernel_launches()
    b.run(40)
    k2 = kernel_launches()
    return ((k2 - k1) - (k1 - k0)) / 20.0


def test_batch_launches_do_not_grow_with_replicas():
    spec = [(256 + 17 * k, 260.0 + 10 * k, 30 + k) for k in range(6)]
    states = [_replica(m, T, seed)[0] for m, T, seed in spec]
    b = BatchReplicas(states)
    b.prepare()
    per_step = _launches_per_step(b)
    one = [_replica(300, 300.0, 99)[0]]
    b1 = BatchReplicas(one)
    b1.prepare()
    per_step_1 = _launches_per_step(b1)
    assert per_step == per_step_1
    assert per_step < 20


def test_batch_thermostats_hold_each_temperature():
    """each replica's Nose-Hoover chain acts on its own temperature"""
    spec = [(300, 260.0, 41), (300, 360.0, 42)]
    states = [_replica(m, T, seed)[0] for m, T, seed in spec]
    b = BatchReplicas(states)
    b.prepare()
    b.run(600)
    temps = []
    for st in states:
        mv2, ndf = st.kinetic()
        temps.append(mv2 * systems.MVV_TO_ENG_REAL / (ndf * systems.BOLTZ_REAL))
        assert st.status()[0] == 0
    assert np.all(np.isfinite(temps))
    assert 150 < temps[0] < 600 and 200 < temps[1] < 700, temps
    assert temps[1] > temps[0], temps


def test_autotune_picks_a_team_and_keeps_the_trajectory():
    """the autotuner times each team size from the initial state and leaves
    the batch prepared from that state: the run that follows matches the
    replicas run one at a time"""
    spec = [(256, 270.0, 51), (333, 330.0, 52)]
    states = [_replica(m, T, seed)[0] for m, T, seed in spec]
    b = BatchReplicas(states)
    best, ms = b.autotune(steps=10, teams=(4, 8, 16))
    assert best in (4, 8, 16) and ms > 0
    b.run(25)
    for (m, T, seed), st in zip(spec, states):
        ref, _ = _replica(m, T, seed)
        IntegratorVerlet(ref).run(25)
        d = np.abs(st.getAtoms()[0] - ref.getAtoms()[0]).max()
        assert d < 1e-3, d
        assert st.status()[0] == 0
