"""Learned E3B three-body surrogate: features, MLP inference and the
hand-written backward pass against the CPU restatement in
oracle/surrogate_ref.py; then training on frames the exact E3B kernel
labels, scored against the exact kernel's three-body forces on frames it was not
trained on, against the method without it (no three-body force)."""
import numpy as np
import pytest

from md_engine_b200 import IntegratorVerlet, systems
from oracle import surrogate_ref as SR

pytestmark = pytest.mark.gpu


def _water(nside=8, seed=5, T=298.0):
    sysd = systems.water_tip4p2005(nside=nside, seed=seed, T=T)
    st, fx = systems.build_water_state(sysd, rcut=6.5, skin=1.0, grid=32, e3b=True, T=T)
    return sysd, st, fx


def test_features_and_frames_match_oracle():
    sysd, st, fx = _water()
    st.prepare()
    st.buildNeighborlists(force=True)
    x, _, _ = st.getAtoms()
    M = len(sysd.molecules)
    raw, fr = fx["e3b"].surrogateFeatures(M)
    ref, F = SR.features(x, np.asarray(sysd.molecules), sysd.L)
    assert np.abs(fr - F).max() < 2e-5
    err = np.abs(raw - ref)
    assert err.max() < 5e-4 * max(1.0, np.abs(ref).max()), err.max()
    assert np.abs(ref).max() > 0.5  # non-trivial environment


def test_mlp_inference_and_gradient_match_oracle():
    sysd, st, fx = _water(nside=6)
    st.prepare()
    rng = np.random.default_rng(3)
    w = np.zeros(SR.N_PARAMS, np.float32)
    for k, (o, s) in SR.OFF.items():
        fan = SR.N_IN if k == "W1" else SR.N_HID
        w[o:o + s] = rng.uniform(-1, 1, s) * (np.sqrt(6.0 / fan) if k.startswith("W") else 0.1)
    e3 = fx["e3b"]
    e3.surrogateSetParams(w, np.zeros(SR.N_IN), np.ones(SR.N_IN), 1.0)
    x = rng.standard_normal((256, SR.N_IN)).astype(np.float32)
    t = np.zeros((256, SR.N_OUT), np.float32)
    t[:, :9] = rng.standard_normal((256, 9))
    y = e3.surrogateInfer(x)
    yr, _, _ = SR.mlp_forward(w, x)
    assert np.abs(y[:, :9] - yr[:, :9]).max() < 2e-2 * np.abs(yr[:, :9]).max()
    loss, g = e3.surrogateGrad(x, t)
    lr, gr = SR.mlp_loss_grad(w, x, t)
    assert loss == pytest.approx(lr, rel=1e-2)
    rel = np.linalg.norm(g - gr) / np.linalg.norm(gr)
    assert rel < 2e-2, rel
    for k, (o, s) in SR.OFF.items():
        if k == "b4":
            continue
        rk = np.linalg.norm(g[o:o + s] - gr[o:o + s]) / max(np.linalg.norm(gr[o:o + s]), 1e-12)
        assert rk < 5e-2, (k, rk)


def test_surrogate_learns_three_body_forces():
    """frames from NVT runs at 260 and 360 K train the network; a frame of a
    third run at 300 K that it never saw scores it against the exact kernel"""
    sysd, st0, fx0 = _water(nside=8, seed=31, T=260.0)
    e30 = fx0["e3b"]
    it0 = IntegratorVerlet(st0)
    it0.run(100)  # relax the lattice
    for _ in range(30):
        it0.run(10)
        e30.surrogateCollect()
    # frames of the 360 K run, labelled through the first state (same topology)
    _, st1, _ = _water(nside=8, seed=32, T=360.0)
    it1 = IntegratorVerlet(st1)
    it1.run(100)
    for _ in range(30):
        it1.run(10)
        xx, vv, _ = st1.getAtoms()
        st0.putAtoms(xx, vv)
        st0.buildNeighborlists(force=True)
        e30.surrogateCollect()
    assert e30.surrogateDatasetSize() == 60 * 512
    l0, l1 = e30.surrogateTrain(3000, batch=1024, lr=2e-3, seed=7)
    assert l1 < 0.5 * l0
    _, st2, _ = _water(nside=8, seed=77, T=300.0)
    IntegratorVerlet(st2).run(150)
    xx, vv, _ = st2.getAtoms()
    st0.putAtoms(xx, vv)
    st0.buildNeighborlists(force=True)
    rmse, rms = e30.surrogateEval()
    # without the network the three-body force is simply missing: error = rms
    assert rms > 0
    ratio = rmse / rms
    print(f"three-body force RMSE / RMS on a held-out frame: {ratio:.4f} (without the surrogate: 1.0)")
    assert ratio < 0.6, ratio


def test_surrogate_drives_the_fused_step():
    sysd, st, fx = _water(nside=6, seed=9)
    it = IntegratorVerlet(st)
    it.run(20)
    e3 = fx["e3b"]
    for _ in range(8):
        it.run(5)
        e3.surrogateCollect()
    e3.surrogateTrain(300, batch=512, lr=2e-3, seed=3)
    e3.surrogateEnable(True)
    it.run(100)
    assert st.status()[0] == 0
    mv2, ndf = st.kinetic()
    T = mv2 * systems.MVV_TO_ENG_REAL / (ndf * systems.BOLTZ_REAL)
    assert 150 < T < 1200
    e3.surrogateEnable(False)
    it.run(10)
    assert st.status()[0] == 0
