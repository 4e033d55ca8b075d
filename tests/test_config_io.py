"""Configuration IO (WriteConfig.cpp, ReadConfig.cpp) on the host: the
files the library writes are taken apart here with the standard library
(xml.etree, base64, struct) -- an independent decoder of the reference's
layout -- and read back into fresh states.  No GPU: a state that was never
prepared keeps its atoms on the host."""
import base64
import os
import struct
import xml.etree.ElementTree as ET

import numpy as np
import pytest

from md_engine_b200 import (Bounds, FixLJCHARMM, FixLJCut, FixLJCutFS, FixRigid, MdxError, State, Vector,
                            WriteConfig, systems)


def _lj_state(n=40, seed=3, turn=1234):
    rng = np.random.default_rng(seed)
    st = State()
    st.units.setLJ()
    L = np.array([7.5, 8.25, 9.0])
    st.bounds = Bounds(st, lo=Vector(-1.0, 0.5, 2.0), hi=Vector(-1.0 + L[0], 0.5 + L[1], 2.0 + L[2]))
    st.rCut = 2.5
    st.padding = 0.4
    st.dt = 0.005
    st.turn = turn
    st.atomParams.addSpecies(handle="A", mass=1.0)
    st.atomParams.addSpecies(handle="B", mass=2.5)
    x = np.array([-1.0, 0.5, 2.0]) + rng.random((n, 3)) * L
    types = rng.integers(0, 2, n)
    q = rng.normal(size=n)
    st.addAtoms(["A" if t == 0 else "B" for t in types], x, q)
    v = rng.normal(size=(n, 3))
    st.setVelocities(np.arange(n), v)
    return st, x, v, types, q


def _b64(node, dtype, width):
    assert node.get("base64") == "1"
    raw = base64.b64decode(node.text.split()[-1])
    a = np.frombuffer(raw, dtype=dtype)
    return a.reshape(-1, width) if width > 1 else a


def test_base64_layout_decodes_with_the_standard_library(tmp_path):
    st, x, v, types, q = _lj_state()
    w = WriteConfig(st, fn=str(tmp_path / "conf"), handle="w", format="base64", writeEvery=1)
    w.write()
    w.finish()
    root = ET.parse(tmp_path / "conf.xml").getroot()
    assert root.tag == "data"
    (cfg,) = list(root)
    assert cfg.tag == "configuration"
    assert cfg.get("turn") == "1234" and cfg.get("numAtoms") == "40" and cfg.get("dimension") == "3"
    assert cfg.get("periodic") == "111"
    assert (cfg.get("rCut"), cfg.get("padding"), cfg.get("dt")) == ("2.500000", "0.400000", "0.005000")
    b = cfg.find("bounds")
    got = [struct.unpack("<d", base64.b64decode(b.get(k)))[0] for k in ("xlo", "ylo", "zlo", "xhi", "yhi", "zhi")]
    assert got == [-1.0, 0.5, 2.0, 6.5, 8.75, 11.0]
    ap = cfg.find("atomParams")
    assert ap.get("numTypes") == "2"
    assert ap.find("handle").text.split() == ["A", "B"]
    assert [float(m) for m in ap.find("mass").text.split()] == [1.0, 2.5]
    np.testing.assert_array_equal(_b64(cfg.find("position"), "<f8", 3), x)
    np.testing.assert_array_equal(_b64(cfg.find("velocity"), "<f8", 3), v)
    np.testing.assert_array_equal(_b64(cfg.find("force"), "<f8", 3), 0.0)
    np.testing.assert_array_equal(_b64(cfg.find("groupTag"), "<u4", 1), 1)
    np.testing.assert_array_equal(_b64(cfg.find("type"), "<i4", 1), types)
    np.testing.assert_array_equal(_b64(cfg.find("id"), "<i4", 1), np.arange(40))
    np.testing.assert_array_equal(_b64(cfg.find("q"), "<f8", 1), q)
    gi = cfg.find("groupInfo")
    assert gi.find("groupHandles").text.split() == ["all"] and gi.find("groupBits").text.split() == ["1"]
    assert cfg.find("molecules") is not None and len(cfg.find("molecules")) == 0
    # the tag order of writeXMLfileBase64 (WriteConfig.cpp:115-155)
    assert [c.tag for c in cfg] == ["bounds", "atomParams", "position", "velocity", "force", "groupTag", "type",
                                    "id", "q", "groupInfo", "molecules"]


def test_base64_round_trip_restores_the_state_bit_for_bit(tmp_path):
    st, x, v, types, q = _lj_state()
    st.createGroup("left", [i for i in range(40) if i % 3 == 0])
    st.createMolecule([0, 1, 2])
    w = WriteConfig(st, fn=str(tmp_path / "rt"), handle="w", format="base64", writeEvery=1)
    w.write()
    w.finish()
    r = State()
    r.rCut = 9.0  # overwritten by the read, as ReadConfig::read does
    r.readConfig.loadFile(str(tmp_path / "rt.xml"))
    assert r.readConfig.next() is True
    assert r.nAtoms == 40 and int(r.turn) == 1234
    assert (r.rCut, r.padding, r.dt) == (2.5, 0.4, 0.005)
    assert r.atomParams.handles == ["A", "B"] and r.atomParams.masses == [1.0, 2.5]
    assert list(r.bounds.lo.v) == [-1.0, 0.5, 2.0] and list(r.bounds.hi.v) == [6.5, 8.75, 11.0]
    xr, vr, fr = r.getAtoms()
    np.testing.assert_array_equal(xr, x)
    np.testing.assert_array_equal(vr, v)
    assert r.groupTagFromHandle("left") == st.groupTagFromHandle("left") == 2
    # write again: identical bytes
    w2 = WriteConfig(r, fn=str(tmp_path / "rt2"), handle="w", format="base64", writeEvery=1)
    w2.write()
    w2.finish()
    assert open(tmp_path / "rt.xml").read() == open(tmp_path / "rt2.xml").read()
    assert r.readConfig.next() is False


def test_single_file_holds_many_configurations_next_prev_moveby(tmp_path):
    st, x, v, types, q = _lj_state(n=12)
    w = WriteConfig(st, fn=str(tmp_path / "traj"), handle="w", format="base64", writeEvery=5)
    turns = [0, 5, 10, 15]
    for t in turns:
        st.turn = t
        w.write()
    w.finish()
    text = open(tmp_path / "traj.xml").read()
    assert text.startswith("<data>\n") and text.endswith("</data>\n")
    assert text.count("<configuration ") == 4
    r = State()
    rc = r.readConfig
    rc.loadFile(str(tmp_path / "traj.xml"))
    seen = []
    while rc.next():
        seen.append(int(r.turn))
    assert seen == turns
    r2 = State()
    r2.readConfig.loadFile(str(tmp_path / "traj.xml"))
    assert r2.readConfig.prev() and int(r2.turn) == 15
    assert r2.readConfig.prev() and int(r2.turn) == 10
    assert r2.readConfig.moveBy(-2) and int(r2.turn) == 0
    assert r2.readConfig.moveBy(3) and int(r2.turn) == 15
    assert not r2.readConfig.moveBy(1)
    r3 = State()
    r3.readConfig.loadFile(str(tmp_path / "traj.xml"))
    assert r3.readConfig.moveBy(2) and int(r3.turn) == 5  # the first move lands on the first configuration


def test_star_in_the_name_writes_one_file_per_turn(tmp_path):
    st, *_ = _lj_state(n=8)
    w = WriteConfig(st, fn=str(tmp_path / "snap*"), handle="w", format="xml", writeEvery=1)
    for t in (0, 7):
        st.turn = t
        w.write()
    w.finish()
    for t in (0, 7):
        root = ET.parse(tmp_path / f"snap{t}.xml").getroot()
        assert root.tag == "data" and root[0].get("turn") == str(t)


def _water_state(nside=2, seed=5):
    sysd = systems.water_tip4p2005(nside=nside, seed=seed)
    st, fx = systems.build_water_state(sysd, rcut=6.0, skin=1.0, grid=32, thermostat=False)
    return sysd, st, fx


def test_plain_xml_carries_the_fix_restart_chunks(tmp_path):
    sysd, st, fx = _water_state()
    w = WriteConfig(st, fn=str(tmp_path / "w"), handle="w", format="xml", writeEvery=1)
    w.write()
    w.finish()
    cfg = ET.parse(tmp_path / "w.xml").getroot()[0]
    assert cfg.find("bounds").get("base64") == "0"
    fixes = {f.get("type"): f for f in cfg.find("fixes")}
    assert set(fixes) == {"LJCut", "ChargeEwald", "Rigid"}
    lj = fixes["LJCut"]
    assert lj.get("handle") == "cut"
    params = {p.get("handle"): np.array([float(t) for t in p.text.split()]) for p in lj.findall("parameter")}
    assert [p.get("handle") for p in lj.findall("parameter")] == ["eps", "rCut", "sig"]  # map order
    # 9 significant digits: the FP32 table value comes back exactly
    assert np.float32(params["sig"][0]) == np.float32(systems.SIG_OO)
    assert np.float32(params["eps"][0]) == np.float32(systems.EPS_OO)
    assert np.all(params["rCut"] == -1000)  # never set: DEFAULT_FILL
    rg = fixes["Rigid"]
    aim = rg.find("atomsInMolecule")
    rows = np.array(aim.text.split(), int).reshape(-1, 4)
    assert int(aim.get("n")) == len(sysd.molecules)
    np.testing.assert_array_equal(rows, np.asarray(sysd.molecules))
    assert rg.find("style").get("type") == "TIP4P/2005" and rg.find("model").get("fourSite") == "true"
    x = np.array(cfg.find("position").text.split(), float).reshape(-1, 3)
    np.testing.assert_allclose(x, st.getAtoms()[0], atol=5e-7)  # "%f"
    # a new state: the fixes created after the read take their chunk
    r = State()
    r.readConfig.loadFile(str(tmp_path / "w.xml"))
    assert r.readConfig.next()
    lj2 = FixLJCut(r, "cut")
    assert lj2.getParameter("sig", "OW", "OW") == pytest.approx(systems.SIG_OO, rel=1e-7)
    assert lj2.getParameter("eps", "OW", "HY") == 0.0
    assert lj2.getParameter("rCut", "OW", "OW") == -1000.0
    other = FixLJCut(r, "other")  # another handle: nothing read
    assert other.getParameter("sig", "OW", "OW") == -1000.0
    rig = FixRigid(r, "rigid", "TIP3P")  # the style is the restart's
    r.activateFix(lj2)
    r.activateFix(rig)
    w2 = WriteConfig(r, fn=str(tmp_path / "w2"), handle="w", format="xml", writeEvery=1)
    w2.write()
    w2.finish()
    cfg2 = ET.parse(tmp_path / "w2.xml").getroot()[0]
    f2 = {f.get("type"): f for f in cfg2.find("fixes")}
    assert ET.tostring(f2["Rigid"]) == ET.tostring(fixes["Rigid"])
    assert ET.tostring(f2["LJCut"]) == ET.tostring(lj)


def test_restart_chunks_of_the_other_pair_styles(tmp_path):
    st, *_ = _lj_state(n=6)
    ch = FixLJCHARMM(st, "ch")
    ch.setParameter("eps", "A", "A", 1.25)
    ch.setParameter("sig14", "A", "B", 0.75)
    fs = FixLJCutFS(st, "fs")
    fs.setParameter("rCut", "B", "B", 2.0)
    st.activateFix(ch)
    w = WriteConfig(st, fn=str(tmp_path / "p"), handle="w", format="xml", writeEvery=1)
    w.write()
    w.finish()
    st.deactivateFix(ch)
    st.activateFix(fs)
    w = WriteConfig(st, fn=str(tmp_path / "q"), handle="w", format="xml", writeEvery=1)
    w.write()
    w.finish()
    c1 = ET.parse(tmp_path / "p.xml").getroot()[0].find("fixes")[0]
    assert c1.get("type") == "LJCHARMM"
    assert [p.get("handle") for p in c1.findall("parameter")] == ["eps", "eps14", "rCut", "sig", "sig14"]
    c2 = ET.parse(tmp_path / "q.xml").getroot()[0].find("fixes")[0]
    assert c2.get("type") == "LJCutFS"
    assert [p.get("handle") for p in c2.findall("parameter")] == ["FCutHandle", "eps", "rCut", "sig"]
    for fn, make, checks in (("p.xml", FixLJCHARMM, [("eps", "A", "A", 1.25), ("sig14", "B", "A", 0.75)]),
                             ("q.xml", FixLJCutFS, [("rCut", "B", "B", 2.0), ("eps", "A", "A", -1000.0)])):
        r = State()
        r.readConfig.loadFile(str(tmp_path / fn))
        assert r.readConfig.next()
        f = make(r, "ch" if make is FixLJCHARMM else "fs")
        for p, a, b, val in checks:
            assert f.getParameter(p, a, b) == val


def test_xyz_and_lammpstrj_trajectories(tmp_path):
    st, x, v, types, q = _lj_state(n=10, turn=40)
    st.createGroup("g", [1, 4, 7])
    w = WriteConfig(st, fn=str(tmp_path / "t"), handle="x", format="xyz", writeEvery=1)
    w.writingVelocities = True
    w.write()
    w.write()
    w.finish()
    lines = open(tmp_path / "t.xyz").read().splitlines()
    assert len(lines) == 2 * 12
    assert lines[0] == "10" and lines[1] == "bounds lo (-1, 0.5, 2) hi (6.5, 8.75, 11)"
    row = lines[2].split()
    assert int(row[0]) == types[0]  # atomic numbers unset (-1): the type
    np.testing.assert_allclose([float(t) for t in row[1:4]], x[0], rtol=1e-5)
    np.testing.assert_allclose([float(t) for t in row[4:7]], v[0], rtol=1e-5)
    lw = WriteConfig(st, fn=str(tmp_path / "t"), handle="l", format="lammpstrj", writeEvery=1, groupHandle="g")
    lw.write()
    lw.finish()
    L = open(tmp_path / "t.lammpstrj").read().splitlines()
    assert L[:4] == ["ITEM: TIMESTEP", "40", "ITEM: NUMBER OF ATOMS", "3"]
    assert L[4] == "ITEM: BOX BOUNDS pp pp pp" and L[5].split() == ["-1", "6.5"]
    assert L[8] == "ITEM: ATOMS id type x y z"
    assert [int(r.split()[0]) for r in L[9:]] == [1, 4, 7]


def test_xyz_guesses_atomic_numbers_in_real_units(tmp_path):
    sysd, st, fx = _water_state(nside=1)
    w = WriteConfig(st, fn=str(tmp_path / "wat"), handle="x", format="xyz", writeEvery=1)
    w.write()
    w.finish()
    rows = open(tmp_path / "wat.xyz").read().splitlines()[2:]
    # the massless M site has no element, so every row carries its type
    assert {r.split()[0] for r in rows} == {"0", "1", "2"}


def test_unwrap_molecules_makes_each_molecule_whole(tmp_path):
    sysd, st, fx = _water_state(nside=2)
    L = sysd.L
    x = np.array(sysd.pos, float)
    o, h1, h2, m = sysd.molecules[0]
    shift = L[0] - (x[o, 0] - sysd.lo[0]) - 0.05  # put O 0.05 A below the upper x face ...
    for a in (o, h1, h2, m):
        x[a, 0] += shift
    x[:, 0] = sysd.lo[0] + np.mod(x[:, 0] - sysd.lo[0], L[0])  # ... and wrap the molecule's atoms apart
    st2, _ = systems.build_water_state(systems.System(**{**sysd.__dict__, "pos": x}), rcut=6.0, skin=1.0,
                                       grid=32, thermostat=False)
    for mol in sysd.molecules:
        st2.createMolecule(list(mol))
    w = WriteConfig(st2, fn=str(tmp_path / "u"), handle="u", format="base64", writeEvery=1, unwrapMolecules=True)
    w.write()
    w.finish()
    xs = _b64(ET.parse(tmp_path / "u.xml").getroot()[0].find("position"), "<f8", 3)
    for mol in sysd.molecules:
        d = xs[list(mol)] - xs[mol[0]]
        assert np.abs(d).max() < 1.5
        com = (xs[list(mol)] * np.array([15.9994, 1.008, 1.008, 0.0])[:, None]).sum(0) / 18.0154
        assert np.all(com >= sysd.lo - 1e-9) and np.all(com < sysd.lo + L + 1e-9)
    raw = np.asarray(st2.getAtoms()[0])
    assert np.abs(raw[h1, 0] - raw[o, 0]) > L[0] / 2 or np.abs(raw[h2, 0] - raw[o, 0]) > L[0] / 2


def test_hand_written_file_plain_numbers_quotes_comments(tmp_path):
    doc = """<?xml version="1.0"?>
<!-- a configuration written by hand -->
<data>
<configuration turn='7' numAtoms='2' dimension='3' periodic='111' rCut='3.0' padding='0.5' dt='0.002'>
<bounds base64='0' xlo='0' ylo='0' zlo='0' xhi='10' yhi='10' zhi='10'/>
<atomParams numTypes='1'><handle> X </handle><mass> 4.0 </mass></atomParams>
<position>1 2 3
4 5 6</position>
<velocity>0 0 0 0.5 0 0</velocity>
<force>0 0 0 0 0 0</force>
<groupTag>1 1</groupTag>
<type>0 0</type>
<id>1 0</id>
<q>0.25 -0.25</q>
</configuration>
</data>
"""
    p = tmp_path / "hand.xml"
    p.write_text(doc)
    r = State()
    r.readConfig.loadFile(str(p))
    assert r.readConfig.next()
    x, v, _ = r.getAtoms()
    np.testing.assert_array_equal(x, [[4, 5, 6], [1, 2, 3]])  # placed by id
    np.testing.assert_array_equal(v, [[0.5, 0, 0], [0, 0, 0]])
    assert r.atomParams.handles == ["X"] and int(r.turn) == 7


@pytest.mark.parametrize("bad,msg", [
    ("<id>0 0</id>", "atom ids"),
    ("<q base64='1'>@@@@</q>", "base64"),
    ("<type>0 3</type>", "type"),
])
def test_reader_rejects_bad_data(tmp_path, bad, msg):
    good = {"id": "<id>0 1</id>", "q": "<q>0 0</q>", "type": "<type>0 0</type>"}
    tag = bad[1:bad.index(" ") if " " in bad[:bad.index(">")] else bad.index(">")]
    good[tag] = bad
    doc = ("<data><configuration turn='0' numAtoms='2' dimension='3' periodic='111' rCut='3' padding='0.5' "
           "dt='0.002'><bounds base64='0' xlo='0' ylo='0' zlo='0' xhi='9' yhi='9' zhi='9'/>"
           "<atomParams numTypes='1'><handle>X</handle><mass>1</mass></atomParams>"
           "<position>0 0 0 1 1 1</position><velocity>0 0 0 0 0 0</velocity><force>0 0 0 0 0 0</force>"
           f"<groupTag>1 1</groupTag>{good['type']}{good['id']}{good['q']}</configuration></data>")
    p = tmp_path / "bad.xml"
    p.write_text(doc)
    r = State()
    r.readConfig.loadFile(str(p))
    with pytest.raises(MdxError, match=msg):
        r.readConfig.next()


def test_reader_rejects_malformed_xml_and_two_dimensions(tmp_path):
    p = tmp_path / "m.xml"
    p.write_text("<data><configuration turn='0'></data>")
    with pytest.raises(MdxError, match="parsed with errors"):
        State().readConfig.loadFile(str(p))
    p.write_text("<data><configuration turn='0' numAtoms='0' dimension='2' periodic='110' rCut='1' padding='1' "
                 "dt='1'/></data>")
    r = State()
    r.readConfig.loadFile(str(p))
    with pytest.raises(MdxError, match="two-dimensional"):
        r.readConfig.next()
    with pytest.raises(MdxError, match="no configuration file"):
        State().readConfig.next()
    assert not os.path.exists(tmp_path / "never.xml")
