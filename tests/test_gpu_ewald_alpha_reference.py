"""The P3M splitting parameter: the oracle's secant (oracle.p3m_alpha, the
restatement the library's host code is checked against to 1e-9 on CPU)
against the reference's own FixChargeEwald::find_optimal_parameters
(FixChargeEwald.cu:918-967) compiled from source (oracle/_ref/librefewald.so).
The solve is host code, but the fix's device arrays initialise the CUDA
runtime when it is constructed, so this runs where a GPU is.

In the reference's precision (float box sides, mesh spacings, cutoff, total
squared charge and alpha) the oracle reproduces the reference's alpha bit
for bit; in FP64, the library's precision, to 1e-6 relative.  The oracle's
FP64 influence function (oracle.p3m_green) against the reference's
Green_function_cu kernel, run by the same harness on the GPU, to 3e-6 of
its largest value."""
import numpy as np
import pytest

from oracle import oracle as O
from oracle import refkernels as R

pytestmark = pytest.mark.gpu

if not R.ewald_available():
    pytest.skip("oracle/_ref/librefewald.so not built", allow_module_level=True)

QQR = O.REAL_UNITS["qqr_to_eng"]
Q2_TIP4P = QQR * (2 * 0.5564 ** 2 + 1.1128 ** 2)  # per molecule

# (natoms, box sides, mesh, cutoff, order, total squared charge)
CASES = [
    (16384, (49.6, 49.6, 49.6), (64, 64, 64), 9.0, 5, 4096 * Q2_TIP4P),   # rigid water, 4,096 molecules
    (2048, (24.83, 24.83, 24.83), (32, 32, 32), 6.5, 5, 512 * Q2_TIP4P),  # rigid water, 512 molecules
    (6000, (30.0, 35.5, 41.25), (32, 32, 64), 10.0, 3, 1500 * Q2_TIP4P),
    (864, (12.7, 12.7, 12.7), (32, 32, 32), 5.0, 1, 216 * Q2_TIP4P),
    (100000, (101.3, 99.7, 100.9), (128, 128, 128), 12.0, 5, 25000 * Q2_TIP4P),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"n{c[0]}_o{c[4]}")
def test_alpha_matches_reference(case):
    natoms, L, sz, rc, order, q2 = case
    a_ref, err = R.ewald_alpha(natoms, L, sz, rc, order, q2)
    assert np.isfinite(err) and err > 0
    a_rf = O.p3m_alpha(None, natoms, L, sz, rc, order, ref_float=True, q2=q2)
    assert a_rf == a_ref
    a64 = O.p3m_alpha(None, natoms, L, sz, rc, order, q2=q2)
    assert a64 == pytest.approx(a_ref, rel=1e-6)


GREEN_CASES = [
    ((24.83, 24.83, 24.83), (32, 32, 32), 5),
    ((49.6, 49.6, 49.6), (64, 64, 64), 5),
    ((30.0, 35.5, 41.25), (32, 32, 64), 3),
]


@pytest.mark.parametrize("case", GREEN_CASES, ids=lambda c: f"{c[1][0]}x{c[1][1]}x{c[1][2]}_o{c[2]}")
def test_green_function_matches_reference_kernel(case):
    """the oracle's FP64 influence function (the one the library's P3M is
    checked against) vs the reference's Green_function_cu, a float kernel
    built with fast math, at the alpha the reference chooses for that box;
    the tolerance is relative to the largest value (measured on a B200: at
    most 1.1e-6 of it, and 3.6e-5 relative wherever |G| is above 1e-3 of
    it)"""
    L, sz, order = case
    natoms = int(round(L[0] * L[1] * L[2] * 0.1334))  # TIP4P/2005 sites at 1 g/cm^3
    alpha, _ = R.ewald_alpha(natoms, L, sz, 9.0, order, natoms / 4 * Q2_TIP4P)
    g_ref = R.ewald_green(L, sz, alpha, order).astype(np.float64)
    g_orc = O.p3m_green(L, sz, alpha, order)
    scale = np.abs(g_orc).max()
    assert scale > 0 and g_ref[0, 0, 0] == 0.0
    np.testing.assert_allclose(g_ref, g_orc, rtol=0, atol=GREEN_TOL * scale)


GREEN_TOL = 3e-6
