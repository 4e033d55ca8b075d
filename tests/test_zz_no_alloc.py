"""mdx_kinetic_noalloc: the allocation-free variant of the FP64 kinetic-energy
sum, for host programs that cannot allocate device memory while they run
(a host serving all device memory from its own pool, or a loop that must not
pay cudaMalloc/cudaFree's implicit synchronisation).  Called through the C
ABI and checked against mdx_kinetic on two calls in a row.  Kept in its own
file, collected last, so a stop-at-first-failure run has already run every
other test if this one fails."""
import ctypes

import pytest

pytestmark = pytest.mark.gpu


def _noalloc(st):
    from md_engine_b200._lib import check, lib
    out = ctypes.c_double()
    check(lib().mdx_kinetic_noalloc(st._h, ctypes.byref(out)))
    return out.value


def test_kinetic_noalloc_matches_allocating_entry_point():
    from md_engine_b200 import IntegratorVerlet, systems
    from tests.helpers import water_small
    sysd = water_small(seed=41)
    st, _ = systems.build_water_state(sysd, rcut=6.5, skin=1.0, grid=32, thermostat=True)
    it = IntegratorVerlet(st)
    it.run(5)
    for _ in range(2):  # two calls in a row share (and reuse) the fixed scratch
        ref, _ = st.kinetic()
        got = _noalloc(st)
        assert ref > 0
        assert abs(got - ref) <= 1e-12 * abs(ref)
        it.run(3)  # different velocities for the second pair of calls
    # a smaller state after a larger one: stale partials beyond its blocks are never read
    small = systems.lj_fcc(ncell=6, seed=2)
    st2, _ = systems.build_lj_state(small, rcut=2.5, skin=0.3)
    st2.prepare()
    ref2, _ = st2.kinetic()
    assert abs(_noalloc(st2) - ref2) <= 1e-12 * abs(ref2)


def test_kinetic_noalloc_rejects_unprepared_state():
    from md_engine_b200 import MdxError, State
    st = State()
    with pytest.raises(MdxError) as e:
        _noalloc(st)
    assert e.value.code == 3
