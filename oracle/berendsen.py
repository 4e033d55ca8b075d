"""Restatement of FixPressureBerendsen's box dilation -- TEST
INFRASTRUCTURE ONLY (nothing in the package imports it).

FixPressureBerendsen::stepFinal (FixPressureBerendsen.cu:26-46): at the
instantaneous scalar pressure p the box scales by
    (1 - dt / period * (target - p) / bulkModulus) ** (1/3)
clamped to [1 - maxDilation, 1 + maxDilation] (defaults bulkModulus 10,
maxDilation 1e-5, FixPressureBerendsen.cu:8-12).

Pinned against the reference's own stepFinal compiled from source on the
CPU (oracle/ref_berendsen_harness.cu -> oracle/_ref/librefbarostat.so;
fixture tests/golden/ref_barostat.json): in the reference's precision
(ref_float: a float time step, State.h:117, and the factor handed to
Mod::scaleSystem as a float real3) bit for bit, NaN included."""
from __future__ import annotations

import numpy as np


def dilation(target, pressure, period, dt, bulk=10.0, max_dil=1e-5, ref_float=False):
    """the box scale factor of one Berendsen step.

    FP64 (the library's precision): a negative base of the cube root (a
    pressure far above the target) is taken as the lower clamp.  ref_float
    (the reference's own behaviour): the time step is a float and the result
    is rounded to float; a negative base gives NaN, which the clamp's
    comparisons let through."""
    lower, upper = 1.0 - max_dil, 1.0 + max_dil
    if ref_float:
        dt = float(np.float32(dt))
    base = 1.0 - dt / period * (target - pressure) / bulk
    if base < 0.0:
        if ref_float:
            return float(np.float32(np.nan))
        return lower
    d = base ** (1.0 / 3.0)
    if d < lower:
        d = lower
    elif d > upper:
        d = upper
    return float(np.float32(d)) if ref_float else d
