"""Host-buffer runs (mdx_integrator_run_host, the call the end-to-end
benchmark makes): positions and velocities by atom id in from FP64 host
arrays, steps, positions/velocities/forces by id out.  Two identical states
are advanced the same way, one through the device-resident run and one
through the host-buffer call fed its own current state: the outputs agree to
the last bits that the P3M spread's float-atomic order leaves free.  A
host-buffer call fed a displaced input must continue from that input."""
import numpy as np
import pytest

from md_engine_b200 import IntegratorVerlet, systems

pytestmark = pytest.mark.gpu


def _state(seed=11):
    sysd = systems.water_tip4p2005(nside=8, seed=seed)
    st, _ = systems.build_water_state(sysd, rcut=9.0, skin=1.0, grid=32)
    return st


def test_run_host_matches_device_run():
    a, b = _state(), _state()
    ia, ib = IntegratorVerlet(a), IntegratorVerlet(b)
    ia.run(20)
    ib.run(20)
    x0, v0, _ = b.getAtoms()
    ia.run(10)
    xa, va, fa = a.getAtoms()
    out = ib.runHost(10, positions=x0, velocities=v0)
    assert set(out) == {"pos", "vel", "force"}
    for k, ref in (("pos", xa), ("vel", va), ("force", fa)):
        assert out[k].shape == ref.shape and out[k].dtype == np.float64
        scale = np.max(np.abs(ref)) + 1e-30
        assert np.max(np.abs(out[k] - ref)) <= 1e-4 * scale, k
    # the state itself moved on: what getAtoms reports is what came out
    xb, vb, fb = b.getAtoms()
    assert np.array_equal(xb, out["pos"]) and np.array_equal(vb, out["vel"]) and np.array_equal(fb, out["force"])


def test_run_host_takes_the_given_input():
    a = _state()
    it = IntegratorVerlet(a)
    it.run(20)
    x0, v0, _ = a.getAtoms()
    # zero velocities in, zero steps: the state takes them exactly (FP32
    # round trip of values that came out of FP32)
    out = it.runHost(0, positions=x0, velocities=np.zeros_like(v0))
    assert np.array_equal(out["pos"], x0)
    assert np.array_equal(out["vel"], np.zeros_like(v0))
    _, v1, _ = a.getAtoms()
    assert np.array_equal(v1, np.zeros_like(v0))
