"""C-ABI boundary tests that need no GPU: the library loads, exports every
entry point declared in include/mdx.h, and rejects bad input with the
documented status codes (no compute calls are made here)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "mdx.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mdx_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from md_engine_b200 import _lib
    lib = _lib.lib()
    names = _declared()
    assert len(names) > 50
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (mdx_[a-z0-9_]+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    for n in names:
        assert hasattr(lib, n)
    # the Python binding covers every declared entry point
    bound = {n for n, _, _ in _lib.SIGNATURES}
    assert set(names) <= bound, sorted(set(names) - bound)


def test_error_codes_without_gpu():
    from md_engine_b200 import Bounds, FixChargeEwald, FixE3B, FixLJCut, FixRigid, MdxError, State, Vector
    st = State()
    with pytest.raises(MdxError) as e:
        st.atomParams.addSpecies("A", -1.0, 1)
    assert e.value.code == 1
    st.atomParams.addSpecies("A", 1.0, 1)
    with pytest.raises(MdxError):
        st.atomParams.addSpecies("A", 1.0, 1)  # duplicate handle
    with pytest.raises(MdxError):
        st.addAtom("B", Vector(0, 0, 0))  # unknown species
    with pytest.raises(MdxError):
        st.bounds = Bounds(st, lo=Vector(0, 0, 0), hi=Vector(-1, 1, 1))
    ew = FixChargeEwald(st, "ew", "all")
    with pytest.raises(MdxError):
        ew.setParameters(48, 48, 48, 9.0, 5)  # only 2^N grids (FixChargeEwald.cu:976-987)
    with pytest.raises(MdxError) as e:
        ew.setParameters(64, 64, 64, 9.0, 3)
    assert e.value.code == 5
    with pytest.raises(MdxError):
        FixE3B(st, "e", "E3B4")
    with pytest.raises(MdxError):
        FixRigid(st, "r", "TIP5P")
    lj = FixLJCut(st, "lj")
    with pytest.raises(MdxError):
        lj.setParameter("bogus", "A", "A", 1.0)
    with pytest.raises(MdxError):
        lj.setParameter("eps", "A", "Z", 1.0)
    # stage calls before prepare are state errors, not crashes
    with pytest.raises(MdxError) as e:
        st.computeForces()
    assert e.value.code == 3


def test_rigid_mass_order_check():
    from md_engine_b200 import FixRigid, MdxError, State
    st = State()
    st.units.setReal()
    st.atomParams.addSpecies("OW", 15.9994, 8)
    st.atomParams.addSpecies("HY", 1.008, 1)
    st.atomParams.addSpecies("OM", 0.0, 0)
    st.addAtoms(["HY", "OW", "HY", "OM"], np.zeros((4, 3)))
    r = FixRigid(st, "r", "TIP4P/2005")
    with pytest.raises(MdxError):
        r.createRigid(0, 1, 2, 3)  # H first: FixRigid.cu:1580-1594 requires O, H, H, M
    r.createRigid(1, 0, 2, 3)


def test_state_attributes_roundtrip():
    from md_engine_b200 import State
    st = State()
    st.rCut = 9.0
    st.padding = 1.0
    st.dt = 2.0
    st.periodicInterval = 7
    assert st.rCut == 9.0 and st.padding == 1.0 and st.dt == 2.0 and st.periodicInterval == 7


def test_product_path_has_no_oracle_import():
    """the package never imports the oracle (fails loudly instead)"""
    pkg = os.path.join(ROOT, "md_engine_b200")
    for root, _, files in os.walk(pkg):
        for f in files:
            if f.endswith(".py"):
                txt = open(os.path.join(root, f)).read()
                assert "import oracle" not in txt and "from oracle" not in txt, f


def test_batch_argument_errors_without_gpu():
    """batch entry points reject bad input before touching the device"""
    from md_engine_b200 import _lib
    lib = _lib.lib()
    b = ctypes.c_void_p()
    assert lib.mdx_batch_create(ctypes.byref(b)) == 0
    assert lib.mdx_batch_add(b, None) == 1
    assert lib.mdx_batch_prepare(b) == 3  # no replicas
    n = ctypes.c_int(-1)
    assert lib.mdx_batch_size(b, ctypes.byref(n)) == 0 and n.value == 0
    st = ctypes.c_void_p()
    assert lib.mdx_state_create(ctypes.byref(st)) == 0
    assert lib.mdx_batch_add(b, st) == 0
    assert lib.mdx_batch_add(b, st) == 1  # the same state twice
    assert lib.mdx_batch_size(b, ctypes.byref(n)) == 0 and n.value == 1
    assert lib.mdx_batch_run_timed(b, 10, 0, 0, None) == 1
    assert lib.mdx_batch_destroy(b) == 0
    assert lib.mdx_state_destroy(st) == 0


def test_surrogate_parameter_count_agrees():
    """the Python binding, the header and the CPU restatement agree on the
    surrogate's parameter blob size (the library writes that many floats)"""
    from md_engine_b200.dash import FixE3B
    from oracle import surrogate_ref
    assert FixE3B.N_PARAMS == surrogate_ref.N_PARAMS == 17616
    assert "17,616 floats" in open(os.path.join(ROOT, "include", "mdx.h")).read()
