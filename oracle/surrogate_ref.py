"""CPU restatement of the learned E3B three-body surrogate -- TEST
INFRASTRUCTURE ONLY (the checker of md_engine_b200/csrc/surrogate.cu; the
surrogate has no reference counterpart, so this restates the library's own
definition: features, frames, and the MLP forward/backward with the same BF16
rounding points).  Only tests/ import it.

  features(): frame e1 = bisector, e2 = (H1 - H2) orthogonalised, e3 = e1 x e2;
      channels O->O, O->H, H1->O, H2->O; shells mu = 2.4 + 0.4 b (O-O, width
      0.4) or 1.5 + 0.5 b (width 0.5); cosine cutoff 5.6 A; per shell
      [sum g, sum g u1, sum g u2, sum g u3] -> feature c*32 + b*4 + k
  mlp_forward / mlp_loss_grad(): 128-64-64-64-16 (9 used), SiLU, BF16
      operands and activations, FP64 accumulation here (FP32 on the GPU)
"""
from __future__ import annotations

import numpy as np

N_IN, N_HID, N_OUT = 128, 64, 16
OFF = {}
_o = 0
for _name, _size in (("W1", N_IN * N_HID), ("b1", N_HID), ("W2", N_HID * N_HID), ("b2", N_HID),
                     ("W3", N_HID * N_HID), ("b3", N_HID), ("W4", N_HID * N_OUT), ("b4", N_OUT)):
    OFF[_name] = (_o, _size)
    _o += _size
N_PARAMS = _o
CUT = 5.6


def bf16(x):
    """round float32 values to bfloat16 (nearest even), returned as float64"""
    a = np.ascontiguousarray(x, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(w):
    w = np.asarray(w, np.float64)
    d = {k: w[o:o + n] for k, (o, n) in OFF.items()}
    d["W1"] = d["W1"].reshape(N_IN, N_HID)
    d["W2"] = d["W2"].reshape(N_HID, N_HID)
    d["W3"] = d["W3"].reshape(N_HID, N_HID)
    d["W4"] = d["W4"].reshape(N_HID, N_OUT)
    return d


def _minimg(d, L):
    return d - L * np.rint(d / L)


def frames(o, h1, h2, L):
    a = _minimg(h1 - o, L)
    b = _minimg(h2 - o, L)
    e1 = a + b
    e1 /= np.linalg.norm(e1, axis=1)[:, None]
    d = a - b
    d -= e1 * np.sum(d * e1, 1)[:, None]
    e2 = d / np.linalg.norm(d, axis=1)[:, None]
    e3 = np.cross(e1, e2)
    return np.stack([e1, e2, e3], 1), o + a, o + b


def features(pos, mol, L):
    """raw features (M x 128) and frames (M x 3 x 3) of rigid water
    molecules mol = [(O, H1, H2, M)] over all other molecules (brute force)"""
    pos = np.asarray(pos, np.float64)
    L = np.asarray(L, np.float64)
    O, H1, H2 = pos[mol[:, 0]], pos[mol[:, 1]], pos[mol[:, 2]]
    F, h1, h2 = frames(O, H1, H2, L)
    M = len(mol)
    out = np.zeros((M, N_IN))
    for m in range(M):
        e = F[m]
        others = np.arange(M) != m
        srcs = (O[m], O[m], h1[m], h2[m])
        tgts = (O[others], np.concatenate([H1[others], H2[others]]), O[others], O[others])
        for c in range(4):
            d = _minimg(tgts[c] - srcs[c], L)
            r = np.linalg.norm(d, axis=1)
            keep = (r < CUT) & (r > 1e-3)
            d, r = d[keep], r[keep]
            u = (d @ e.T) / r[:, None]
            fc = 0.5 * (np.cos(np.pi * r / CUT) + 1.0)
            for b in range(8):
                mu = 2.4 + 0.4 * b if c == 0 else 1.5 + 0.5 * b
                gam = 3.125 if c == 0 else 2.0
                g = np.exp(-gam * (r - mu) ** 2) * fc
                base = c * 32 + b * 4
                out[m, base] = g.sum()
                out[m, base + 1:base + 4] = (g[:, None] * u).sum(0)
    return out, F


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def mlp_forward(w, x):
    """outputs (n x 16), pre-activations and activations; BF16 weights,
    inputs and activations as on the GPU"""
    p = unpack(w)
    a = bf16(x)
    zs, acts = [], [a]
    for l, (W, b) in enumerate((("W1", "b1"), ("W2", "b2"), ("W3", "b3"), ("W4", "b4"))):
        z = a @ bf16(p[W]) + p[b]
        zs.append(z)
        if l < 3:
            a = bf16(silu(z))
            acts.append(a)
    return zs[-1], zs, acts


def mlp_loss_grad(w, x, t):
    """mean squared error over the 9 used outputs and its gradient (flat, the
    parameter blob's order)"""
    p = unpack(w)
    n = len(x)
    y, zs, acts = mlp_forward(w, x)
    d = (y - t)[:, :9]
    loss = float(np.mean(d ** 2))
    dz = np.zeros_like(y)
    dz[:, :9] = 2.0 * d / (n * 9)
    dz = bf16(dz)
    grads = {}
    names = (("W1", "b1"), ("W2", "b2"), ("W3", "b3"), ("W4", "b4"))
    for l in range(3, -1, -1):
        W, b = names[l]
        grads[W] = acts[l].T @ dz
        grads[b] = dz.sum(0)
        if l == 0:
            break
        da = dz @ bf16(p[W]).T
        dz = bf16(da * dsilu(zs[l - 1]))
    flat = np.zeros(N_PARAMS)
    for k, (o, s) in OFF.items():
        flat[o:o + s] = grads[k].reshape(-1)
    return loss, flat
