"""Writers inside a run (Integrator::asyncOperations, Integrator.cu:77-113)
and a restart from the written file, on the GPU path: the configurations land
at the multiples of writeEvery with the device state of that turn, and a
state rebuilt from the restart file (atoms, species, bounds and the fixes'
restart chunks, FixLJCut parameters and FixRigid molecules, read as the
reference's ReadConfig does) continues the trajectory of the original."""
import base64
import xml.etree.ElementTree as ET

import numpy as np
import pytest

from md_engine_b200 import FixChargeEwald, FixLJCut, FixRigid, IntegratorVerlet, State, WriteConfig, systems
from tests.helpers import water_small

pytestmark = pytest.mark.gpu


def _b64(node, dtype, width):
    raw = base64.b64decode(node.text.split()[-1])
    return np.frombuffer(raw, dtype=dtype).reshape(-1, width)


def test_writers_fire_during_a_run_and_a_restart_continues_it(tmp_path):
    sysd = water_small(seed=29)
    st, fx = systems.build_water_state(sysd, rcut=6.5, skin=1.0, grid=32, alpha=0.35, thermostat=False)
    w = WriteConfig(st, fn=str(tmp_path / "run"), handle="w", format="base64", writeEvery=5)
    rs = WriteConfig(st, fn=str(tmp_path / "restart*"), handle="r", format="xml", writeEvery=15)
    st.activateWriteConfig(w)
    st.activateWriteConfig(rs)
    integ = IntegratorVerlet(st)
    integ.run(16)  # writes after the steps of turns 0, 5, 10, 15
    x16, v16, _ = st.getAtoms()
    st.deactivateWriteConfig(w)
    st.deactivateWriteConfig(rs)
    w.finish()
    rs.finish()
    cfgs = list(ET.parse(tmp_path / "run.xml").getroot())
    assert [int(c.get("turn")) for c in cfgs] == [0, 5, 10, 15]
    np.testing.assert_array_equal(_b64(cfgs[-1].find("position"), "<f8", 3), x16)
    np.testing.assert_array_equal(_b64(cfgs[-1].find("velocity"), "<f8", 3), v16)
    assert not np.array_equal(_b64(cfgs[0].find("position"), "<f8", 3), x16)
    assert st.status()[0] == 0

    # restart from the plain-XML file of turn 15, fixes created after the read
    r = State()
    r.readConfig.loadFile(str(tmp_path / "restart15.xml"))
    assert r.readConfig.next() and int(r.turn) == 15
    lj = FixLJCut(r, "cut")
    assert lj.getParameter("sig", "OW", "OW") == pytest.approx(systems.SIG_OO, rel=1e-7)
    ew = FixChargeEwald(r, "charge", "all")
    ew.setParameters(32, 32, 32, 6.5, 5)
    ew.setAlpha(0.35)
    rig = FixRigid(r, "rigid", "TIP4P/2005")
    for f in (lj, ew, rig):
        r.activateFix(f)
    r.periodicInterval = int(st.periodicInterval)
    r.units.setReal()
    IntegratorVerlet(r).run(10)
    # the same start built through the ordinary API from the file's numbers:
    # a restart is a fresh start (prepareForRun runs again, as in the
    # reference), so the two must agree to the float-atomic order
    cfg = ET.parse(tmp_path / "restart15.xml").getroot()[0]
    xf = np.array(cfg.find("position").text.split(), float).reshape(-1, 3)
    vf = np.array(cfg.find("velocity").text.split(), float).reshape(-1, 3)
    b = cfg.find("bounds")  # plain XML: "%f" bounds too
    lo = np.array([float(b.get(k)) for k in ("xlo", "ylo", "zlo")])
    hi = np.array([float(b.get(k)) for k in ("xhi", "yhi", "zhi")])
    fresh = systems.System(**{**sysd.__dict__, "pos": xf, "vel": vf, "lo": lo, "L": hi - lo})
    st2, _ = systems.build_water_state(fresh, rcut=6.5, skin=1.0, grid=32, alpha=0.35, thermostat=False)
    st2.turn = 15
    IntegratorVerlet(st2).run(10)
    xa, xb = st2.getAtoms()[0], r.getAtoms()[0]
    d = xa - xb
    d -= sysd.L * np.rint(d / sysd.L)
    assert np.abs(d).max() < 1e-4, np.abs(d).max()
    assert r.status()[0] == 0 and int(r.turn) == 25
    # and it follows the uninterrupted run (the restart's first half kick,
    # like the reference's, uses forces whose M-site part is not yet moved
    # onto O and H, so the runs part by ~1e-2 A over 10 steps, no more)
    integ.run(10)
    d = st.getAtoms()[0] - xb
    d -= sysd.L * np.rint(d / sysd.L)
    assert np.abs(d).max() < 0.1, np.abs(d).max()
