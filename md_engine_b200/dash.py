"""Python front end mirroring DASH's Python API (python/DASH.cpp:34-131) for
the hot path: State, Bounds, Vector, units, atomParams, FixLJCut, FixWCA,
FixChargeEwald, FixE3B, FixRigid, FixNoseHoover, IntegratorVerlet.

Every call goes through the C ABI of libmdx.so (include/mdx.h); argument
names and meanings follow the reference, e.g.

    state = State()
    state.units.setReal()
    state.bounds = Bounds(state, lo=Vector(0, 0, 0), hi=Vector(L, L, L))
    state.rCut = 9.0; state.padding = 1.0; state.dt = 2.0
    state.atomParams.addSpecies(handle='OW', mass=15.9994, atomicNum=8)
    lj = FixLJCut(state, 'cut'); lj.setParameter('sig', 'OW', 'OW', 3.1589)
    state.activateFix(lj)
    IntegratorVerlet(state).run(1000)
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import P, c_dbl, c_flt, c_i64, c_int, c_u32, c_u64, c_void_p, check, lib

UNITS_REAL = 0
UNITS_LJ = 1


class Vector:
    """3-vector with the arithmetic scripts use (src/Vector.h)."""

    def __init__(self, x=0.0, y=0.0, z=0.0):
        self.v = np.array([float(x), float(y), float(z)])

    def __getitem__(self, i):
        return self.v[i]

    def __add__(self, o):
        return Vector(*(self.v + np.asarray(o.v if isinstance(o, Vector) else o)))

    def __sub__(self, o):
        return Vector(*(self.v - np.asarray(o.v if isinstance(o, Vector) else o)))

    def __mul__(self, s):
        return Vector(*(self.v * s))

    def len(self):
        return float(np.linalg.norm(self.v))

    def __repr__(self):
        return f"Vector({self.v[0]}, {self.v[1]}, {self.v[2]})"


class Bounds:
    def __init__(self, state, lo, hi):
        self.lo = lo if isinstance(lo, Vector) else Vector(*lo)
        self.hi = hi if isinstance(hi, Vector) else Vector(*hi)


class _Units:
    def __init__(self, st):
        self._st = st

    def setReal(self):
        check(lib().mdx_state_set_units(self._st._h, UNITS_REAL))
        self._st._units = UNITS_REAL

    def setLJ(self):
        check(lib().mdx_state_set_units(self._st._h, UNITS_LJ))
        self._st._units = UNITS_LJ


class _AtomParams:
    def __init__(self, st):
        self._st = st
        self.handles = []
        self.masses = []

    def addSpecies(self, handle, mass, atomicNum=-1):
        t = c_int()
        check(lib().mdx_state_add_species(self._st._h, handle.encode(), float(mass), int(atomicNum), ctypes.byref(t)))
        self.handles.append(handle)
        self.masses.append(float(mass))
        return t.value

    def _refresh(self):
        """the species the library holds (after a configuration was read)"""
        n = c_int()
        check(lib().mdx_state_get_species(self._st._h, -1, None, 0, None, None, ctypes.byref(n)))
        self.handles, self.masses = [], []
        buf = ctypes.create_string_buffer(256)
        for k in range(n.value):
            m = c_dbl()
            check(lib().mdx_state_get_species(self._st._h, k, buf, 256, ctypes.byref(m), None, None))
            self.handles.append(buf.value.decode())
            self.masses.append(m.value)

    def typeFromHandle(self, handle):
        return self.handles.index(handle)

    @property
    def numTypes(self):
        return len(self.handles)


def _darr(a, n=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(P(c_dbl))


class _ReadConfig:
    """state.readConfig (src/ReadConfig.cpp): loadFile(fn), then next(),
    prev() or moveBy(n) load a configuration of the file into the state and
    return whether there was one; fixes created afterwards read their restart
    data from that configuration."""

    def __init__(self, st):
        self._st = st
        self.fileOpen = False

    def loadFile(self, fn):
        check(lib().mdx_read_config_load(self._st._h, str(fn).encode()))
        self.fileOpen = True

    def _move(self, op, by=0):
        found = c_int()
        check(lib().mdx_read_config_move(self._st._h, op, int(by), ctypes.byref(found)))
        if found.value:
            self._st._after_read()
        return bool(found.value)

    def next(self):
        return self._move(0)

    def prev(self):
        return self._move(1)

    def moveBy(self, by):
        return self._move(2, by)


class State:
    """src/State.h:63-146 -- owns the atoms and the device copy."""

    _DOUBLE_KEYS = ("rCut", "padding", "dt")
    _INT_KEYS = ("periodicInterval", "nThreadPerAtom", "nThreadPerBlock", "gridStencil", "gridHomeGroup", "turn",
                 "pairForm", "pairBlocksPerSM")

    def __init__(self):
        h = c_void_p()
        check(lib().mdx_state_create(ctypes.byref(h)))
        object.__setattr__(self, "_h", h)
        object.__setattr__(self, "units", _Units(self))
        object.__setattr__(self, "atomParams", _AtomParams(self))
        object.__setattr__(self, "_bounds", None)
        object.__setattr__(self, "_fixes", [])
        object.__setattr__(self, "_units", UNITS_LJ)
        object.__setattr__(self, "_charges", [])
        object.__setattr__(self, "readConfig", _ReadConfig(self))
        object.__setattr__(self, "writeConfigs", [])

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().mdx_state_destroy(h)
            except Exception:
                pass

    def __setattr__(self, k, v):
        if k in self._DOUBLE_KEYS:
            check(lib().mdx_state_set_double(self._h, k.encode(), float(v)))
        elif k in self._INT_KEYS:
            check(lib().mdx_state_set_int(self._h, k.encode(), int(v)))
        elif k == "bounds":
            lo = (ctypes.c_double * 3)(*v.lo.v)
            hi = (ctypes.c_double * 3)(*v.hi.v)
            check(lib().mdx_state_set_bounds(self._h, lo, hi))
            object.__setattr__(self, "_bounds", v)
        else:
            object.__setattr__(self, k, v)

    def __getattr__(self, k):
        if k in State._DOUBLE_KEYS:
            out = c_dbl()
            check(lib().mdx_state_get_double(self._h, k.encode(), ctypes.byref(out)))
            return out.value
        if k in State._INT_KEYS or k in ("nlistCapacity", "cellsPerSide", "molListCapacity", "molListEntries"):
            out = c_i64()
            check(lib().mdx_state_get_int(self._h, k.encode(), ctypes.byref(out)))
            return out.value
        if k == "bounds":
            # the library's box (a barostat or a read configuration moves it)
            if object.__getattribute__(self, "_bounds") is None:
                return None
            lo = (ctypes.c_double * 3)()
            hi = (ctypes.c_double * 3)()
            check(lib().mdx_state_get_bounds(self._h, lo, hi))
            return Bounds(self, lo=Vector(*lo), hi=Vector(*hi))
        raise AttributeError(k)

    def _after_read(self):
        self.atomParams._refresh()
        lo = (ctypes.c_double * 3)()
        hi = (ctypes.c_double * 3)()
        check(lib().mdx_state_get_bounds(self._h, lo, hi))
        object.__setattr__(self, "_bounds", Bounds(self, lo=Vector(*lo), hi=Vector(*hi)))

    # -- configuration IO, groups, molecules --------------------------------
    def activateWriteConfig(self, wc):
        check(lib().mdx_state_activate_write_config(self._h, wc._h))
        if wc not in self.writeConfigs:
            self.writeConfigs.append(wc)
        return True

    def deactivateWriteConfig(self, wc):
        check(lib().mdx_state_deactivate_write_config(self._h, wc._h))
        if wc in self.writeConfigs:
            self.writeConfigs.remove(wc)
        return True

    def createGroup(self, handle, atoms=()):
        ids = np.ascontiguousarray(list(atoms), np.int32)
        check(lib().mdx_state_create_group(self._h, handle.encode(), len(ids), ids.ctypes.data_as(P(c_int))))
        return True

    def groupTagFromHandle(self, handle):
        b = c_u32()
        check(lib().mdx_state_group_tag(self._h, handle.encode(), ctypes.byref(b)))
        return b.value

    def scaleSystem(self, scale):
        """Mod::scaleSystem: the box and the positions scaled by `scale`
        about the box centre (rigid molecules by their centres of mass)"""
        check(lib().mdx_state_scale_system(self._h, float(scale)))
        lo = (ctypes.c_double * 3)()
        hi = (ctypes.c_double * 3)()
        check(lib().mdx_state_get_bounds(self._h, lo, hi))
        object.__setattr__(self, "_bounds", Bounds(self, lo=Vector(*lo), hi=Vector(*hi)))

    def createMolecule(self, ids):
        ids = np.ascontiguousarray(list(ids), np.int32)
        check(lib().mdx_state_create_molecule(self._h, len(ids), ids.ctypes.data_as(P(c_int))))

    def setSpecialNeighborCoefs(self, onetwo, onethree, onefour):
        check(lib().mdx_state_set_special_neighbor_coefs(self._h, onetwo, onethree, onefour))

    # -- atoms ------------------------------------------------------------
    def addAtom(self, handle, pos, q=0.0):
        p = pos.v if isinstance(pos, Vector) else pos
        return self.addAtoms([handle], np.asarray([p], np.float64), np.asarray([q], np.float64))

    def addAtoms(self, handles, positions, charges=None):
        """Bulk State::addAtom; returns the first new id (ids are consecutive)."""
        n = len(handles)
        pos, pp = _darr(np.asarray(positions, np.float64).reshape(n, 3))
        q = np.zeros(n) if charges is None else np.asarray(charges, np.float64)
        q, qp = _darr(q)
        enc = [h.encode() for h in handles]
        arr = (ctypes.c_char_p * n)(*enc)
        first = c_int()
        check(lib().mdx_state_add_atoms(self._h, n, arr, pp, qp, ctypes.byref(first)))
        self._charges.extend(q.tolist())
        return first.value

    @property
    def nAtoms(self):
        n = c_int()
        check(lib().mdx_state_n_atoms(self._h, ctypes.byref(n)))
        return n.value

    def setVelocities(self, ids, vels):
        ids = np.ascontiguousarray(ids, np.int32)
        v, vp = _darr(np.asarray(vels).reshape(len(ids), 3))
        check(lib().mdx_state_set_velocities(self._h, len(ids), ids.ctypes.data_as(P(c_int)), vp))

    def getAtoms(self):
        """(positions, velocities, forces) by atom id, (n,3) float64."""
        n = self.nAtoms
        x = np.zeros((n, 3))
        v = np.zeros((n, 3))
        f = np.zeros((n, 3))
        check(lib().mdx_state_get_atoms(self._h, x.ctypes.data_as(P(c_dbl)), v.ctypes.data_as(P(c_dbl)),
                                        f.ctypes.data_as(P(c_dbl))))
        return x, v, f

    def putAtoms(self, positions=None, velocities=None):
        px = vx = None
        if positions is not None:
            xa, px = _darr(positions)
        if velocities is not None:
            va, vx = _darr(velocities)
        check(lib().mdx_state_put_atoms(self._h, px, vx))

    def activateFix(self, fix):
        check(lib().mdx_state_activate_fix(self._h, fix._h))
        self._fixes.append(fix)

    def deactivateFix(self, fix):
        check(lib().mdx_state_deactivate_fix(self._h, fix._h))
        if fix in self._fixes:
            self._fixes.remove(fix)

    # -- stage-level access (tests, observables) ----------------------------
    def prepare(self):
        check(lib().mdx_prepare(self._h))

    def buildNeighborlists(self, force=True):
        check(lib().mdx_nlist_build(self._h, 1 if force else 0))

    def getNeighborList(self, maxPerAtom=None):
        """Grid.getNeighborList: (counts[id], ids[id, k], tags[id, k]) sorted per id."""
        n = self.nAtoms
        c = np.zeros(n, np.int32)
        if maxPerAtom is None:
            check(lib().mdx_nlist_get(self._h, 0, c.ctypes.data_as(P(c_int)), None, None))
            maxPerAtom = max(int(c.max()) if n else 0, 1)
        nb = np.zeros((n, maxPerAtom), np.int32)
        tg = np.zeros((n, maxPerAtom), np.int32)
        check(lib().mdx_nlist_get(self._h, maxPerAtom, c.ctypes.data_as(P(c_int)), nb.ctypes.data_as(P(c_int)),
                                  tg.ctypes.data_as(P(c_int))))
        return c, nb, tg

    def computeForces(self, virialMode=0):
        check(lib().mdx_compute_forces(self._h, int(virialMode)))

    def potentialEnergy(self):
        """[pair (LJ/WCA + Ewald real), Ewald reciprocal (incl. self), E3B 2-body, E3B 3-body]"""
        out = (ctypes.c_double * 4)()
        check(lib().mdx_potential_energy(self._h, out))
        return np.array(list(out))

    def kinetic(self):
        s = c_dbl()
        n = c_dbl()
        check(lib().mdx_kinetic(self._h, ctypes.byref(s), ctypes.byref(n)))
        return s.value, n.value

    def pressure(self):
        """DataComputerPressure's scalar pressure and the total virial (6) from
        a virial-mode force evaluation at the current positions (forces kept)"""
        p = c_dbl()
        v = (ctypes.c_double * 6)()
        check(lib().mdx_pressure(self._h, ctypes.byref(p), v))
        return p.value, np.array(list(v))

    def virials(self):
        n = self.nAtoms
        per = np.zeros((n, 6))
        tot = (ctypes.c_double * 6)()
        check(lib().mdx_get_virials(self._h, per.ctypes.data_as(P(c_dbl)), tot))
        return per, np.array(list(tot))

    def status(self):
        b = c_u32()
        m = c_u32()
        nb = c_u64()
        check(lib().mdx_state_status(self._h, ctypes.byref(b), ctypes.byref(m), ctypes.byref(nb)))
        return b.value, m.value, nb.value

    def synchronize(self):
        check(lib().mdx_state_synchronize(self._h))

    STAGES = {"pair": 0, "p3m": 1, "e3b": 2, "nlist": 3, "first_half": 4, "second_half": 5, "p3m_spread": 6,
              "p3m_solve": 7, "p3m_gather": 8, "p3m_step": 9}

    def timeStage(self, stage, iters=20, flushBytes=0):
        """average device ms of one launch of a hot-path stage"""
        out = c_dbl()
        check(lib().mdx_time_stage(self._h, self.STAGES[stage], int(iters), int(flushBytes), ctypes.byref(out)))
        return out.value


class _Fix:
    _h = None

    def __del__(self):
        pass  # fixes live as long as their state (the state owns the device data)


class FixPair(_Fix):
    def setParameter(self, param, handleA, handleB, val):
        check(lib().mdx_fix_pair_set_parameter(self._h, param.encode(), handleA.encode(), handleB.encode(), float(val)))

    def getParameter(self, param, handleA, handleB):
        out = c_dbl()
        check(lib().mdx_fix_pair_get_parameter(self._h, param.encode(), handleA.encode(), handleB.encode(),
                                               ctypes.byref(out)))
        return out.value


class FixLJCut(FixPair):
    """FixLJCut(state, handle, mixingRules='geometric') (src/Fixes/FixLJCut.cu:14-28)"""

    def __init__(self, state, handle, mixingRules="geometric"):
        h = c_void_p()
        check(lib().mdx_fix_lj_cut_create(state._h, handle.encode(), mixingRules.encode(), ctypes.byref(h)))
        self._h = h
        self.state = state
        self.handle = handle


class FixWCA(FixPair):
    """FixWCA(state, handle, mixingRules='geometric') (src/Fixes/FixWCA.cu)"""

    def __init__(self, state, handle, mixingRules="geometric"):
        h = c_void_p()
        check(lib().mdx_fix_wca_create(state._h, handle.encode(), mixingRules.encode(), ctypes.byref(h)))
        self._h = h
        self.state = state
        self.handle = handle


def _pair_fix(obj, create, state, handle, mixingRules):
    h = c_void_p()
    check(create(state._h, handle.encode(), mixingRules.encode(), ctypes.byref(h)))
    obj._h = h
    obj.state = state
    obj.handle = handle


class FixLJCutFS(FixPair):
    """FixLJCutFS(state, handle, mixingRules='geometric') (src/Fixes/FixLJCutFS.cu:12-26):
    force-shifted Lennard-Jones; parameters eps, sig, rCut"""

    def __init__(self, state, handle, mixingRules="geometric"):
        _pair_fix(self, lib().mdx_fix_lj_cut_fs_create, state, handle, mixingRules)


class FixLJCHARMM(FixPair):
    """FixLJCHARMM(state, handle, mixingRules='geometric') (src/Fixes/FixLJCHARMM.cu:15-32):
    LJ with 1-4 parameters; parameters eps, sig, eps14, sig14, rCut"""

    def __init__(self, state, handle, mixingRules="geometric"):
        _pair_fix(self, lib().mdx_fix_lj_charmm_create, state, handle, mixingRules)


class FixTICG(FixPair):
    """FixTICG(state, handle, mixingRules='geometric') (src/Fixes/FixTICG.cu:11-22):
    soft-sphere overlap; parameters C and rCut for every pair of species"""

    def __init__(self, state, handle, mixingRules="geometric"):
        _pair_fix(self, lib().mdx_fix_ticg_create, state, handle, mixingRules)


class FixChargePairDSF(_Fix):
    """FixChargePairDSF(state, handle, groupHandle) (src/Fixes/FixChargePairDSF.cu):
    damped shifted force charges, evaluated inside the pair fix's kernel"""

    def __init__(self, state, handle, groupHandle="all"):
        h = c_void_p()
        check(lib().mdx_fix_charge_pair_dsf_create(state._h, handle.encode(), groupHandle.encode(), ctypes.byref(h)))
        self._h = h
        self.state = state

    def setParameters(self, alpha, r_cut):
        check(lib().mdx_fix_charge_pair_dsf_set_parameters(self._h, float(alpha), float(r_cut)))


class FixChargeEwald(_Fix):
    """FixChargeEwald(state, handle, groupHandle) (src/Fixes/FixChargeEwald.cu:828-839)"""

    def __init__(self, state, handle, groupHandle="all"):
        h = c_void_p()
        check(lib().mdx_fix_charge_ewald_create(state._h, handle.encode(), groupHandle.encode(), ctypes.byref(h)))
        self._h = h
        self.state = state

    def setParameters(self, szx, szy=None, szz=None, rcut=-1.0, interpolation_order=5):
        """setParameters(sz, rcut, order) or (szx, szy, szz, rcut, order)."""
        if szy is not None and szz is None:
            rcut, interpolation_order, szy, szz = szy, (rcut if rcut != -1.0 else 5), szx, szx
        if szy is None:
            szy = szz = szx
        check(lib().mdx_fix_charge_ewald_set_parameters(self._h, int(szx), int(szy), int(szz), float(rcut),
                                                        int(interpolation_order)))

    def setAlpha(self, alpha):
        check(lib().mdx_fix_charge_ewald_set_alpha(self._h, float(alpha)))

    @property
    def alpha(self):
        a = c_dbl()
        check(lib().mdx_fix_charge_ewald_get_alpha(self._h, ctypes.byref(a)))
        return a.value


class FixE3B(_Fix):
    """FixE3B(state, handle, style) (src/Fixes/FixE3B.cu:16-36)"""

    def __init__(self, state, handle, style="E3B3"):
        h = c_void_p()
        check(lib().mdx_fix_e3b_create(state._h, handle.encode(), style.encode(), ctypes.byref(h)))
        self._h = h
        self.state = state

    def addMolecule(self, id_O, id_H1, id_H2, id_M):
        check(lib().mdx_fix_e3b_add_molecule(self._h, int(id_O), int(id_H1), int(id_H2), int(id_M)))

    # ---- learned three-body surrogate (no DASH counterpart) ----------------
    N_IN, N_OUT = 128, 16
    N_PARAMS = (128 * 64 + 64) + 2 * (64 * 64 + 64) + (64 * 16 + 16)  # 17,616

    def surrogateCollect(self):
        """append the current frame: features + exact three-body forces"""
        check(lib().mdx_e3b_surrogate_collect(self.state._h, self._h))

    def surrogateDatasetSize(self):
        n = ctypes.c_int64()
        check(lib().mdx_e3b_surrogate_dataset_size(self._h, ctypes.byref(n)))
        return n.value

    def surrogateTrain(self, iters, batch=4096, lr=1e-3, seed=1):
        """(loss of the first, loss of the last minibatch)"""
        a, b = c_dbl(), c_dbl()
        check(lib().mdx_e3b_surrogate_train(self.state._h, self._h, int(iters), int(batch), float(lr), int(seed),
                                            ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def surrogateEnable(self, on=True):
        check(lib().mdx_e3b_surrogate_enable(self._h, 1 if on else 0))

    def surrogateEval(self):
        """(rmse, rms) of the surrogate's three-body forces on the current frame"""
        a, b = c_dbl(), c_dbl()
        check(lib().mdx_e3b_surrogate_eval(self.state._h, self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def surrogateParams(self):
        w = np.zeros(self.N_PARAMS, np.float32)
        mu = np.zeros(self.N_IN, np.float32)
        isd = np.zeros(self.N_IN, np.float32)
        sc = c_flt()
        check(lib().mdx_e3b_surrogate_get_params(self._h, w.ctypes.data_as(P(c_flt)), mu.ctypes.data_as(P(c_flt)),
                                                 isd.ctypes.data_as(P(c_flt)), ctypes.byref(sc)))
        return w, mu, isd, sc.value

    def surrogateSetParams(self, w, mean, inv_std, scale):
        w = np.ascontiguousarray(w, np.float32)
        mean = np.ascontiguousarray(mean, np.float32)
        inv_std = np.ascontiguousarray(inv_std, np.float32)
        check(lib().mdx_e3b_surrogate_set_params(self.state._h, self._h, w.ctypes.data_as(P(c_flt)),
                                                 mean.ctypes.data_as(P(c_flt)), inv_std.ctypes.data_as(P(c_flt)),
                                                 float(scale)))

    def surrogateFeatures(self, nmol):
        raw = np.zeros((nmol, self.N_IN), np.float32)
        fr = np.zeros((nmol, 9), np.float32)
        check(lib().mdx_e3b_surrogate_features(self.state._h, self._h, raw.ctypes.data_as(P(c_flt)),
                                               fr.ctypes.data_as(P(c_flt))))
        return raw, fr.reshape(nmol, 3, 3)

    def surrogateInfer(self, x):
        x = np.ascontiguousarray(x, np.float32)
        y = np.zeros((len(x), self.N_OUT), np.float32)
        check(lib().mdx_e3b_surrogate_infer(self.state._h, self._h, x.ctypes.data_as(P(c_flt)), len(x),
                                            y.ctypes.data_as(P(c_flt))))
        return y

    def surrogateGrad(self, x, t):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        g = np.zeros(self.N_PARAMS, np.float32)
        loss = c_dbl()
        check(lib().mdx_e3b_surrogate_grad(self.state._h, self._h, x.ctypes.data_as(P(c_flt)),
                                           t.ctypes.data_as(P(c_flt)), len(x), g.ctypes.data_as(P(c_flt)),
                                           ctypes.byref(loss)))
        return loss.value, g


class FixRigid(_Fix):
    """FixRigid(state, handle, style) (src/Fixes/FixRigid.cu:18-37)"""

    def __init__(self, state, handle, style="TIP4P/2005"):
        h = c_void_p()
        check(lib().mdx_fix_rigid_create(state._h, handle.encode(), style.encode(), ctypes.byref(h)))
        self._h = h
        self.state = state

    def createRigid(self, id_a, id_b, id_c, id_d=-1):
        check(lib().mdx_fix_rigid_create_rigid(self._h, int(id_a), int(id_b), int(id_c), int(id_d)))

    # single hooks (stage-level parity)
    def savePrev(self):
        check(lib().mdx_rigid_save_prev(self.state._h, self._h))

    def settlePositions(self):
        check(lib().mdx_rigid_settle_positions(self.state._h, self._h))

    def settleVelocities(self):
        check(lib().mdx_rigid_settle_velocities(self.state._h, self._h))

    def distributeMSite(self):
        check(lib().mdx_rigid_distribute_msite(self.state._h, self._h))

    def validateConstraints(self):
        """FixRigid::validateConstraints: the number of molecules whose side
        lengths or bond velocities are off by more than 1e-3 (0 = all fine);
        the C call returns MDX_ERR_NUMERIC when it is not 0"""
        n = c_u32()
        rc = lib().mdx_rigid_validate(self.state._h, self._h, ctypes.byref(n))
        if rc not in (0, 6):
            check(rc)
        return n.value


class FixPressureBerendsen(_Fix):
    """FixPressureBerendsen(state, handle, pressure, period, applyEvery)
    (src/Fixes/FixPressureBerendsen.cu): Berendsen box rescaling every
    applyEvery turns toward `pressure` (state units) with time constant
    `period`."""

    _KEYS = ("maxDilation", "bulkModulus", "pressure", "period")

    def __init__(self, state, handle, pressure, period, applyEvery):
        h = c_void_p()
        check(lib().mdx_fix_pressure_berendsen_create(state._h, handle.encode(), float(pressure), float(period),
                                                      int(applyEvery), ctypes.byref(h)))
        object.__setattr__(self, "_h", h)
        object.__setattr__(self, "handle", handle)
        object.__setattr__(self, "applyEvery", int(applyEvery))

    def setParameters(self, maxDilation=-1):
        if maxDilation > 0:
            check(lib().mdx_fix_pressure_berendsen_set(self._h, b"maxDilation", float(maxDilation)))

    def _get(self, k):
        out = c_dbl()
        check(lib().mdx_fix_pressure_berendsen_get(self._h, k.encode(), ctypes.byref(out)))
        return out.value

    def __setattr__(self, k, v):
        if k in FixPressureBerendsen._KEYS:
            check(lib().mdx_fix_pressure_berendsen_set(self._h, k.encode(), float(v)))
        else:
            object.__setattr__(self, k, v)

    def __getattr__(self, k):
        if k in FixPressureBerendsen._KEYS or k in ("lastPressure", "lastDilation"):
            return self._get(k)
        if k == "applications":
            return int(self._get(k))
        raise AttributeError(k)


class FixNoseHoover(_Fix):
    """FixNoseHoover(state, handle, groupHandle) (src/Fixes/FixNoseHoover.cu:97-130)"""

    def __init__(self, state, handle, groupHandle="all"):
        h = c_void_p()
        check(lib().mdx_fix_nose_hoover_create(state._h, handle.encode(), groupHandle.encode(), ctypes.byref(h)))
        self._h = h
        self.state = state

    def setTemperature(self, temperature, timeConstant):
        check(lib().mdx_fix_nose_hoover_set_temperature(self._h, float(temperature), float(timeConstant)))

    def setPressure(self, pressMode, pressure, timeConstant):
        """FixNoseHoover::setPressure (FixNoseHoover.cu:193-202); pressMode "ISO" """
        check(lib().mdx_fix_nose_hoover_set_pressure(self._h, pressMode.encode(), float(pressure),
                                                     float(timeConstant)))

    def _get(self, k):
        out = c_dbl()
        check(lib().mdx_fix_nose_hoover_get(self._h, k.encode(), ctypes.byref(out)))
        return out.value

    @property
    def lastPressure(self):
        return self._get("lastPressure")

    @property
    def pressVel(self):
        return self._get("pressVel")


class WriteConfig:
    """WriteConfig(state, fn, handle, format, writeEvery, groupHandle='all',
    unwrapMolecules=False) (src/WriteConfig.cpp:389-453): format 'base64',
    'xml', 'xyz' or 'lammpstrj'; a '*' in fn writes one file per turn.  Fires
    during runs once activated with state.activateWriteConfig; write() writes
    the current configuration now."""

    _KEYS = ("writeEvery", "unwrapMolecules", "writingVelocities", "writingForces")

    def __init__(self, state, fn, handle, format, writeEvery, groupHandle="all", unwrapMolecules=False):
        h = c_void_p()
        check(lib().mdx_write_config_create(state._h, str(fn).encode(), handle.encode(), format.encode(),
                                            int(writeEvery), groupHandle.encode(), int(bool(unwrapMolecules)),
                                            ctypes.byref(h)))
        object.__setattr__(self, "_h", h)
        object.__setattr__(self, "state", state)
        object.__setattr__(self, "handle", handle)
        object.__setattr__(self, "format", format)
        object.__setattr__(self, "_vals", {"writeEvery": int(writeEvery), "unwrapMolecules": bool(unwrapMolecules),
                                           "writingVelocities": False, "writingForces": False})

    def __setattr__(self, k, v):
        if k in self._KEYS:
            check(lib().mdx_write_config_set(self._h, k.encode(), int(v)))
            self._vals[k] = type(self._vals[k])(v)
        else:
            object.__setattr__(self, k, v)

    def __getattr__(self, k):
        if k in WriteConfig._KEYS:
            return object.__getattribute__(self, "_vals")[k]
        raise AttributeError(k)

    def write(self):
        check(lib().mdx_write_config_write(self._h, -1))

    def finish(self):
        """close the file (the single-file XML's </data>); the writer is spent"""
        h = object.__getattribute__(self, "_h")
        if h is not None and h.value:
            if self in self.state.writeConfigs:
                self.state.writeConfigs.remove(self)
            lib().mdx_write_config_destroy(h)
            object.__setattr__(self, "_h", c_void_p())

    def __del__(self):
        try:
            self.finish()
        except Exception:
            pass


class IntegratorVerlet:
    """IntegratorVerlet(state).run(numTurns) (src/Integrators/IntegratorVerlet.cu:649-770)."""

    def __init__(self, state):
        h = c_void_p()
        check(lib().mdx_integrator_verlet_create(state._h, ctypes.byref(h)))
        self._h = h
        self.state = state

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().mdx_integrator_destroy(h)
            except Exception:
                pass

    def writeOutput(self):
        """Integrator::writeOutput: every active writer writes now"""
        check(lib().mdx_write_output(self.state._h))

    def setMode(self, mode):
        """0: fused, CUDA-graph captured (default); 1: one kernel per reference hook."""
        check(lib().mdx_integrator_set_mode(self._h, int(mode)))

    def run(self, numTurns):
        out = c_dbl()
        check(lib().mdx_integrator_run(self._h, int(numTurns), ctypes.byref(out)))
        return out.value

    def runHost(self, numTurns, positions=None, velocities=None, want=("pos", "vel", "force")):
        """run with host buffers: copy positions/velocities (by id) in, step,
        copy positions/velocities/forces out -- all inside one C-ABI call."""
        n = self.state.nAtoms

        def inp(a):
            if a is None:
                return None, None
            a = np.ascontiguousarray(a, np.float64).reshape(n, 3)
            return a, a.ctypes.data_as(P(c_dbl))

        pa, pp = inp(positions)
        va, vp = inp(velocities)
        outs = {k: np.empty((n, 3)) for k in want}  # every element is written
        op = [outs[k].ctypes.data_as(P(c_dbl)) if k in outs else None for k in ("pos", "vel", "force")]
        check(lib().mdx_integrator_run_host(self._h, int(numTurns), pp, vp, op[0], op[1], op[2]))
        return outs

    def runTimed(self, numTurns, chunk, flushBytes):
        """device milliseconds summed over chunks (L2 flushed between chunks)"""
        out = c_dbl()
        check(lib().mdx_integrator_run_timed(self._h, int(numTurns), int(chunk), int(flushBytes), ctypes.byref(out)))
        return out.value

    def autotune(self, reps=10, caps=(6, 8, 10, 12, 14, -1)):
        """Integrator::tune's role (Integrator.cu:272-376) for the molecule
        form of all-rigid water: the pair grid's blocks per SM timed against
        the P3M chain and E3B beside it; the fastest is kept on the state.
        (best cap, ms per force phase); (0, 0.0) where there is no such shape."""
        arr = (c_int * len(caps))(*caps)
        best, ms = c_int(), c_dbl()
        check(lib().mdx_integrator_autotune(self._h, int(reps), arr, len(caps), ctypes.byref(best), ctypes.byref(ms)))
        return best.value, ms.value

    # stage-level halves
    def firstHalf(self):
        check(lib().mdx_verlet_first_half(self.state._h))

    def secondHalf(self):
        check(lib().mdx_verlet_second_half(self.state._h))


class BatchReplicas:
    """Independent rigid-water States advanced together, one launch per phase
    for all replicas (no DASH counterpart; each replica keeps
    IntegratorVerlet's per-step semantics).  The states must stay alive while
    the batch exists."""

    def __init__(self, states):
        h = c_void_p()
        check(lib().mdx_batch_create(ctypes.byref(h)))
        self._h = h
        self.states = list(states)
        for st in self.states:
            check(lib().mdx_batch_add(self._h, st._h))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().mdx_batch_destroy(h)
            except Exception:
                pass

    def __len__(self):
        return len(self.states)

    def prepare(self):
        check(lib().mdx_batch_prepare(self._h))

    def run(self, numTurns):
        """device milliseconds of the call"""
        out = c_dbl()
        check(lib().mdx_batch_run(self._h, int(numTurns), ctypes.byref(out)))
        return out.value

    def runTimed(self, numTurns, chunk, flushBytes):
        out = c_dbl()
        check(lib().mdx_batch_run_timed(self._h, int(numTurns), int(chunk), int(flushBytes), ctypes.byref(out)))
        return out.value

    def autotune(self, steps=20, teams=(4, 8, 16, 32)):
        """(best team size, device ms per step); leaves the batch prepared with it"""
        arr = (c_int * len(teams))(*teams)
        best = c_int()
        ms = c_dbl()
        check(lib().mdx_batch_autotune(self._h, int(steps), arr, len(teams), ctypes.byref(best), ctypes.byref(ms)))
        return best.value, ms.value


def kernel_launches():
    return int(lib().mdx_kernel_launch_count())
