"""ctypes wrappers for the parity checker.  TEST INFRASTRUCTURE ONLY.

  Oracle     -- liboracle.so, the FP64 C restatement (remd_oracle.c)
  Reference  -- oracle/_ref/libremdref*.so, the reference's own CPU sources
                compiled unmodified around ref_driver.cxx

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs import this
module.  Nothing under remd_b200/ does.
"""
from __future__ import annotations

import ctypes as C
import os
import shutil
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
NUM_AVG = 19
AVG_NAMES = ["LJ", "CLMB", "WALL", "VOL", "TRA", "ROT", "T", "P", "Px", "Py", "Pz",
             "TOT", "DRF", "TSTs", "TSTv", "BSTx", "BSTy", "BSTz", "DUMMY"]

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def _ptr(a, t=_dp):
    return a.ctypes.data_as(t) if a is not None else None


def build_oracle():
    """Compile liboracle.so (and the reference libraries when the reference
    sources are present) with oracle/Makefile."""
    targets = ["liboracle.so"]
    if os.path.isdir(os.environ.get("REMD_REFERENCE", "/root/reference") + "/src"):
        targets.append("ref")
    env = dict(os.environ)
    if "REMD_REFERENCE" in os.environ:
        env["REF"] = os.environ["REMD_REFERENCE"]
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True, env=env)


# ---------------------------------------------------------------- data model
import sys as _sys
_sys.path.insert(0, os.path.dirname(HERE))
from remd_b200.inputs import (MolType, ReplicaState, SystemSpec, read_chk,  # noqa: E402,F401
                              read_moltype)


# ---------------------------------------------------------------- oracle (C restatement)
class _OrcMolType(C.Structure):
    _fields_ = [("nsite", C.c_int), ("body", C.c_double * 15), ("mass", C.c_double * 5),
                ("sgm2", C.c_double * 25), ("eps", C.c_double * 25), ("q", C.c_double * 5),
                ("inertia", C.c_double * 3)]


class _OrcSystem(C.Structure):
    _fields_ = [("nmol", C.c_int), ("tconstant", C.c_int), ("pconstant", C.c_int),
                ("confined", C.c_int), ("dt", C.c_double), ("dthalf", C.c_double),
                ("rcut", C.c_double), ("rswitch", C.c_double), ("nfwall", C.c_int),
                ("wall_length_param", C.c_double), ("wall_length", C.c_double),
                ("fwall", _dp), ("mt", _OrcMolType)]


class _OrcReplica(C.Structure):
    _fields_ = [("r", _dp), ("v", _dp), ("q", _dp), ("p", _dp), ("f", _dp), ("n", _dp),
                ("m", _dp), ("I", _dp), ("ar", _dp), ("af", _dp),
                ("s", C.c_double), ("Ps", C.c_double), ("Q", C.c_double),
                ("Pv", C.c_double * 3), ("W", C.c_double), ("L", C.c_double * 3),
                ("T", C.c_double), ("P", C.c_double), ("gkT", C.c_double), ("H0", C.c_double),
                ("pot", C.c_double), ("lj", C.c_double), ("clmb", C.c_double),
                ("wall", C.c_double), ("vir", C.c_double * 3),
                ("tra3", C.c_double * 3), ("tra", C.c_double), ("rot", C.c_double),
                ("kin", C.c_double), ("Tk", C.c_double), ("prs", C.c_double * 4),
                ("tsm", C.c_double), ("tsp", C.c_double), ("tst", C.c_double),
                ("bst", C.c_double), ("tot", C.c_double), ("ham", C.c_double),
                ("npairs", C.c_longlong)]


_ORC = None


def _orc_lib():
    global _ORC
    if _ORC is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build_oracle()
        lib = C.CDLL(path)
        for name in ["orc_unit_time", "orc_unit_temp", "orc_unit_press", "orc_unit_coulomb",
                     "orc_unit_mass"]:
            getattr(lib, name).restype = C.c_double
        lib.orc_volume.restype = C.c_double
        lib.orc_replica_exchange.restype = C.c_int
        _ORC = lib
    return _ORC


def units():
    lib = _orc_lib()
    return dict(time=lib.orc_unit_time(), temp=lib.orc_unit_temp(), press=lib.orc_unit_press(),
                coulomb=lib.orc_unit_coulomb(), mass=lib.orc_unit_mass())


def wall_table(confined, nfwall, wall_length, sgm, eps, rho):
    out = np.zeros(2 * nfwall)
    _orc_lib().orc_wall_table(C.c_int(confined), C.c_int(nfwall), C.c_double(wall_length),
                              C.c_double(sgm), C.c_double(eps), C.c_double(rho), _ptr(out))
    return out.reshape(nfwall, 2)


class Oracle:
    """One replica advanced by the C restatement."""

    def __init__(self, spec: SystemSpec, state: ReplicaState, fwall=None):
        lib = _orc_lib()
        self.lib, self.spec = lib, spec
        mt = spec.moltype
        self._mt = _OrcMolType()
        lib.orc_moltype_from_input(C.byref(self._mt), C.c_int(mt.nsite),
                                   _ptr(np.ascontiguousarray(mt.r, dtype=float)),
                                   _ptr(mt.mass), _ptr(mt.sigma), _ptr(mt.eps), _ptr(mt.charge))
        self.sys = _OrcSystem()
        lib.orc_system_init(C.byref(self.sys), spec.nmol, spec.tconstant, spec.pconstant,
                            spec.confined, C.c_double(spec.dt), C.c_double(spec.rcut),
                            C.c_double(spec.rswitch), spec.nfwall, C.c_double(spec.wall_length))
        self.sys.mt = self._mt
        if spec.confined:
            self.fwall = (np.ascontiguousarray(fwall, dtype=float).reshape(-1) if fwall is not None
                          else wall_table(spec.confined, spec.nfwall, spec.wall_length,
                                          spec.sgm_wall, spec.eps_wall, spec.rho_wall).reshape(-1))
            self.sys.fwall = _ptr(self.fwall)
        n, ns = spec.nmol, mt.nsite
        self.r = np.ascontiguousarray(state.r, dtype=float).copy()
        self.v = np.ascontiguousarray(state.v, dtype=float).copy()
        self.q = np.ascontiguousarray(state.q, dtype=float).copy()
        self.p = np.ascontiguousarray(state.p, dtype=float).copy()
        self.f = np.zeros((n, 3))
        self.n = np.zeros((n, 4))
        self.m = np.ascontiguousarray(state.m, dtype=float).copy()
        self.I = np.ascontiguousarray(state.I, dtype=float).copy()
        self.ar = np.zeros((n * ns, 3))
        self.af = np.zeros((n * ns, 3))
        rep = _OrcReplica()
        for k in ["r", "v", "q", "p", "f", "n", "m", "I", "ar", "af"]:
            setattr(rep, k, _ptr(getattr(self, k)))
        rep.s, rep.Ps, rep.Q, rep.W = state.s, state.Ps, state.Q, state.W
        for d in range(3):
            rep.Pv[d] = state.Pv[d]
            rep.L[d] = state.L[d]
        rep.T, rep.P = state.T, state.P
        rep.gkT = 6.0 * n * state.T
        self.rep = rep

    # state access
    def state(self) -> ReplicaState:
        r = self.rep
        return ReplicaState(self.r.copy(), self.v.copy(), self.q.copy(), self.p.copy(),
                            self.m.copy(), self.I.copy(), r.s, r.Ps, r.Q, np.array(r.Pv[:]),
                            r.W, np.array(r.L[:]), r.T, r.P)

    def force(self):
        self.lib.orc_force(C.byref(self.sys), C.byref(self.rep))

    def initialize_property(self):
        self.lib.orc_initialize_property(C.byref(self.sys), C.byref(self.rep))

    def steps(self, n):
        self.lib.orc_execute_steps(C.byref(self.sys), C.byref(self.rep), C.c_int(n))

    def calc_properties(self):
        self.lib.orc_calc_properties(C.byref(self.sys), C.byref(self.rep))

    def average(self):
        out = np.zeros(NUM_AVG)
        self.lib.orc_get_average(C.byref(self.sys), C.byref(self.rep), _ptr(out))
        return out

    def volume(self):
        return self.lib.orc_volume(C.byref(self.sys), C.byref(self.rep))

    def velocity_scaling(self):
        self.lib.orc_velocity_scaling(C.byref(self.sys), C.byref(self.rep))

    def ang_velocity_scaling(self):
        self.lib.orc_ang_velocity_scaling(C.byref(self.sys), C.byref(self.rep))

    def kill_momentum(self):
        self.lib.orc_kill_momentum(C.byref(self.sys), C.byref(self.rep))

    def change_temperature(self, T):
        self.lib.orc_change_temperature(C.byref(self.sys), C.byref(self.rep), C.c_double(T))

    def apply_condition(self, T, P):
        self.lib.orc_apply_condition(C.byref(self.sys), C.byref(self.rep), C.c_double(T),
                                     C.c_double(P))

    def set_tstat_mass(self, Q):
        self.rep.Q, self.rep.s, self.rep.Ps = Q, 1.0, 0.0

    def set_TP(self, T, P):
        self.rep.T, self.rep.P = T, P
        self.rep.gkT = 6.0 * self.spec.nmol * T

    def prop(self):
        r = self.rep
        return dict(pot=r.pot, lj=r.lj, clmb=r.clmb, wall=r.wall, vir=np.array(r.vir[:]),
                    tra=r.tra, rot=r.rot, kin=r.kin, tot=r.tot, ham=r.ham, H0=r.H0,
                    gkT=r.gkT, s=r.s, Ps=r.Ps, Pv=np.array(r.Pv[:]), L=np.array(r.L[:]),
                    npairs=r.npairs)


def exchange_lists(ntemp, npress):
    cap = max(ntemp * npress // 2, 1)
    lists = np.zeros(8 * cap, dtype=np.int32)
    ln = np.zeros(4, dtype=np.int32)
    _orc_lib().orc_exchange_lists(ntemp, npress, _ptr(lists, _ip), _ptr(ln, _ip))
    lists = lists.reshape(4, cap, 2)
    return [lists[t, :ln[t]].copy() for t in range(4)]


def conditions_geometrical(ntemp, npress, tmin, tmax, pmin, pmax):
    n = ntemp * npress
    T, P = np.zeros(n), np.zeros(n)
    _orc_lib().orc_conditions_geometrical(ntemp, npress, C.c_double(tmin), C.c_double(tmax),
                                          C.c_double(pmin), C.c_double(pmax), _ptr(T), _ptr(P))
    return T, P


def replica_exchange(ntemp, npress, pconstant, step, index, T, P, pot, vol, u):
    """One REMD::ReplicaExchange (in place on index/T/P).  Returns accepted flags."""
    acc = np.zeros(max(ntemp * npress // 2, 1), dtype=np.int32)
    isx = np.zeros(ntemp * npress, dtype=np.uint8)
    n = _orc_lib().orc_replica_exchange(
        ntemp, npress, pconstant, C.c_long(step), _ptr(index, _ip), _ptr(T), _ptr(P),
        _ptr(np.ascontiguousarray(pot, dtype=float)), _ptr(np.ascontiguousarray(vol, dtype=float)),
        _ptr(np.ascontiguousarray(u, dtype=float)), _ptr(acc, _ip),
        isx.ctypes.data_as(C.POINTER(C.c_ubyte)))
    return acc[:n].copy()


# ---------------------------------------------------------------- compiled reference
_REFLIBS = {}


def gro_atoms(mol_name, atom_names, r, q, L, body):
    """IOManager::ConvertMoleculesToAtoms (src/io_manager.cxx:797-814): per site,
    molecule id i+1, the names padded as MakeMolTypeList pads them
    (src/molecules.cxx:86, 95), atom id, coordinates (r L + R(q) b) in nm.
    r (n,3) box fractions, q (n,4), L (3,) and body (k,3) in A."""
    from remd_b200.systems import body_to_space
    n, k = len(r), len(body)
    mname = mol_name.ljust(5)
    anames = [a.rjust(5) for a in atom_names]
    sites = body_to_space(np.asarray(q, dtype=float), np.asarray(body, dtype=float))   # (n,k,3)
    coor = (np.asarray(r, dtype=float)[:, None, :] * np.asarray(L, dtype=float) + sites) * 0.1
    molid = np.repeat(np.arange(1, n + 1), k)
    return molid, [mname] * (n * k), anames * n, np.arange(1, n * k + 1), coor.reshape(-1, 3)


def gro_text(molid, molname, atomname, atomid, coor, L, comment="test"):
    """write_gro_file (src/gro.cxx:118-135) as text: comment, atom count, one
    "%5d%s%s%5d%8.3f%8.3f%8.3f%8.4f%8.4f%8.4f" line per atom (velocities 0),
    the box "%10.5f%10.5f%10.5f"."""
    out = [comment, "%5d" % len(molid)]
    for m, mn, an, a, c in zip(molid, molname, atomname, atomid, coor):
        out.append("%5d%s%s%5d%8.3f%8.3f%8.3f%8.4f%8.4f%8.4f" % (m, mn, an, a, c[0], c[1], c[2],
                                                               0.0, 0.0, 0.0))
    out.append("%10.5f%10.5f%10.5f" % tuple(L))
    return "\n".join(out) + "\n"


def cdv_text(r, q, L, body, T, P, confined, wall_length):
    """One replica's snapshot as REMDGPU::OutputCDV writes it (src/remdgpu.cu:700-804),
    from its GPU state: the centre as the fixed-point box fraction (int)(2^32 (r-1/2))
    (src/remdgpu.cu:261-263), box and wall length as float, site offsets from the
    device M2A in double (src/remdgpu.cu:2607-2634, body coordinates as float) rounded
    to float, each printed as float(centre) * float(L 2^-32) + offset.  T, P reduced,
    held as float (cond0).  Numbers in the C++ stream default format (%g)."""
    from remd_b200.inputs import UNIT_PRESS, UNIT_TEMP
    f32 = np.float32
    g = lambda x: "%g" % float(x)  # noqa: E731
    Lf = np.asarray(L, dtype=f32)
    wl = f32(wall_length)
    lo = [-0.5 * float(Lf[d]) for d in range(3)]
    hi = [0.5 * float(Lf[d]) for d in range(3)]
    if confined == 1:
        lo[0] = lo[1] = -float(wl)
        hi[0] = hi[1] = float(wl)
    elif confined == 2:
        lo[2], hi[2] = -0.5 * float(wl), 0.5 * float(wl)
    head = "'" + "".join(" box_s%s=%s" % (a, g(v)) for a, v in zip("xyz", lo))
    head += "".join(" box_e%s=%s" % (a, g(v)) for a, v in zip("xyz", hi))
    head += (" r0=1.0 r1=0.8 r2=0.8 c0=(1.0,0.0,0.0) c1=(1.0,1.0,1.0) c2=(1.0,1.0,1.0)"
             " bond0_c=(1.0,1.0,1.0)")
    Tk = float(f32(T)) * UNIT_TEMP
    Pp = float(f32(P)) * UNIT_PRESS
    head += ' st0="T=%s K, P=%s MPa" st0_pos=(-2.0,-2.0)' % (g(Tk), g(Pp / 1e6))
    lines = [head]
    itof = Lf * f32(2.0 ** -32)
    b = np.asarray(body, dtype=f32).astype(float)
    for i in range(len(r)):
        gi = [int(4294967296.0 * (float(r[i][d]) - 0.5)) for d in range(3)]
        x, y, z, w = (float(v) for v in q[i])
        sx, sy, sz, sw = x * x, y * y, z * z, w * w
        xy, xz, xw = 2 * x * y, 2 * x * z, 2 * x * w
        yz, yw, zw = 2 * y * z, 2 * y * w, 2 * z * w
        for k in range(len(b)):
            bx, by, bz = b[k]
            ar = ((sx + sy - sz - sw) * bx + (yz - xw) * by + (yw + xz) * bz,
                  (yz + xw) * bx + (sx - sy + sz - sw) * by + (zw - xy) * bz,
                  (yw - xz) * bx + (zw + xy) * by + (sx - sy - sz + sw) * bz)
            pos = [f32(f32(gi[d]) * itof[d]) + f32(ar[d]) for d in range(3)]
            lines.append("%d %d %s %s %s" % (i, k, g(pos[0]), g(pos[1]), g(pos[2])))
    return "\n".join(lines) + "\n"


class Histograms:
    """REMDInfo's (volume, potential) histograms, one per condition slot
    (src/remdinfo.h:93-139, 299-331; 500 x 500 bins, linear sampling), fed as
    REMD::IncrementHistogram feeds them (src/remd.cxx:803-813) and written as
    REMDInfo::OutputHistogram writes them (src/remdinfo.cxx:723-758)."""
    NB = 500

    def __init__(self, nslot, energy_min, energy_max, volume_min, volume_max):
        self.emin, self.emax, self.vmin, self.vmax = energy_min, energy_max, volume_min, volume_max
        self.de = (energy_max - energy_min) / float(self.NB)
        self.dv = (volume_max - volume_min) / float(self.NB)
        self.hist = np.zeros((nslot, self.NB, self.NB), dtype=np.int64)
        self.ave = np.zeros((nslot, self.NB, self.NB, 19))
        self.bounds = np.zeros((nslot, 5), dtype=np.int64)   # vmin vmax pmin pmax samples

    def increment(self, index, avg, nmol):
        """index[slot] = replica at that condition; avg (nrep, 19) GetAverages rows."""
        for c, ind in enumerate(index):
            a = avg[ind]
            pot = (a[0] + a[1] + a[2]) / float(nmol)
            vol = a[3] / float(nmol)
            if vol < self.vmin or vol >= self.vmax or pot < self.emin or pot >= self.emax:
                raise ValueError("potential energy or volume is not in the histogram range")
            v = int((vol - self.vmin) / self.dv)
            p = int((pot - self.emin) / self.de)
            b = self.bounds[c]
            if b[4] == 0:
                b[0] = b[1] = v
                b[2] = b[3] = p
            b[0], b[1] = min(b[0], v), max(b[1], v)
            b[2], b[3] = min(b[2], p), max(b[3], p)
            b[4] += 1
            self.hist[c, v, p] += 1
            self.ave[c, v, p] += a

    def text(self, c):
        b = self.bounds[c]
        out = ["#vmax vmin pmax pmin", "# %d %d %d %d" % (b[1], b[0], b[3], b[2])]
        for v in range(b[0], b[1] + 1):
            vol = self.vmin + v * self.dv
            for p in range(b[2], b[3] + 1):
                pot = self.emin + p * self.de
                n = int(self.hist[c, v, p])
                avg = self.ave[c, v, p] / n if n > 0 else np.zeros(19)
                out.append(" %10.6e %10.6e %10d" % (vol, pot, n) + "".join(" %10.6e" % x for x in avg))
            out.append("")
        return "\n".join(out) + "\n"

    @staticmethod
    def file_name(directory, P, T):
        return "%s/histo_P%f_T%f.dat" % (directory, P, T)


def reference_write_gro(path, molid, molname, atomname, atomid, coor, L, comment="test"):
    """The reference's own write_gro_file (src/gro.cxx:118-135, compiled into
    oracle/_ref) on the same atoms."""
    lib = _ref_lib()
    n = len(molid)
    enc = lambda xs: (C.c_char_p * n)(*[x.encode() for x in xs])  # noqa: E731
    mi = np.ascontiguousarray(molid, dtype=np.int32)
    ai = np.ascontiguousarray(atomid, dtype=np.int32)
    cc = np.ascontiguousarray(coor, dtype=float)
    LL = np.ascontiguousarray(L, dtype=float)
    lib.ref_write_gro(path.encode(), C.c_int(n), _ptr(mi, _ip), enc(molname), enc(atomname),
                      _ptr(ai, _ip), _ptr(cc), _ptr(LL), comment.encode())


def reference_available(variant="generic"):
    return os.path.exists(_ref_path(variant))


def _ref_path(variant):
    name = {"generic": "libremdref.so", "tuned4": "libremdref_tuned4.so",
            "shipped": "libremdref_shipped.so", "slitwall": "libremdref_slitwall.so"}[variant]
    return os.path.join(REF_DIR, name)


def _ref_lib(variant="generic"):
    if variant not in _REFLIBS:
        lib = C.CDLL(_ref_path(variant))
        lib.ref_create.restype = C.c_void_p
        lib.ref_create.argtypes = [C.c_char_p]
        lib.ref_remdinfo_create.restype = C.c_void_p
        lib.ref_remdinfo_create.argtypes = [C.c_char_p]
        for fn in ["ref_destroy", "ref_initialize_property", "ref_calc_force",
                   "ref_calc_properties", "ref_update_hamiltonian", "ref_velocity_scaling",
                   "ref_ang_velocity_scaling", "ref_kill_momentum"]:
            getattr(lib, fn).argtypes = [C.c_void_p]
        for fn in ["ref_set_temperature", "ref_set_pressure", "ref_set_tstat_mass",
                   "ref_change_temperature"]:
            getattr(lib, fn).argtypes = [C.c_void_p, C.c_double]
        lib.ref_execute_steps.argtypes = [C.c_void_p, C.c_int]
        lib.ref_execute_steps_parallel.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_int, C.c_int]
        lib.ref_remdinfo_exchange.restype = C.c_int
        lib.ref_remdinfo_exchange.argtypes = [C.c_void_p, C.c_long, _dp, _dp, _dp, _ip]
        lib.ref_remdinfo_arrays.argtypes = [C.c_void_p, _ip, _dp, _dp]
        lib.ref_remdinfo_set_arrays.argtypes = [C.c_void_p, _ip, _dp, _dp]
        lib.ref_remdinfo_increment_histogram.argtypes = [C.c_void_p, _dp, _dp, _dp]
        lib.ref_remdinfo_output_histogram.argtypes = [C.c_void_p]
        lib.ref_remdinfo_read_histogram.argtypes = [C.c_void_p]
        lib.ref_write_gro.argtypes = [C.c_char_p, C.c_int, _ip, C.POINTER(C.c_char_p),
                                      C.POINTER(C.c_char_p), _ip, _dp, _dp, C.c_char_p]
        lib.ref_write_chk.argtypes = [C.c_void_p, C.c_char_p]
        for fn in ["ref_set_state", "ref_get_state", "ref_get_property", "ref_get_average",
                   "ref_get_fwall", "ref_get_property_line"]:
            getattr(lib, fn).argtypes = None
        _REFLIBS[variant] = lib
    return _REFLIBS[variant]


class Reference:
    """One replica held by the reference's own Molecules object."""

    def __init__(self, spec: SystemSpec, state: ReplicaState, moltype_path, variant="generic"):
        lib = _ref_lib(variant)
        self.lib, self.spec = lib, spec
        # the reference's slit wall table is also written to ./force.dat
        # (src/force_calculator.cxx:164): build it in a scratch directory
        cwd, tmp = os.getcwd(), tempfile.mkdtemp()
        try:
            os.chdir(tmp)
            self.h = C.c_void_p(lib.ref_create(spec.inp_text(moltype_path).encode()))
        finally:
            os.chdir(cwd)
            shutil.rmtree(tmp, ignore_errors=True)
        st = state
        lib.ref_set_state(self.h, _ptr(np.ascontiguousarray(st.r, float)),
                          _ptr(np.ascontiguousarray(st.v, float)),
                          _ptr(np.ascontiguousarray(st.q, float)),
                          _ptr(np.ascontiguousarray(st.p, float)),
                          _ptr(np.ascontiguousarray(st.m, float)),
                          _ptr(np.ascontiguousarray(st.I, float)),
                          C.c_double(st.s), C.c_double(st.Ps), C.c_double(st.Q),
                          _ptr(np.ascontiguousarray(st.Pv, float)), C.c_double(st.W),
                          _ptr(np.ascontiguousarray(st.L, float)))
        lib.ref_set_temperature(self.h, st.T)
        lib.ref_set_pressure(self.h, st.P)

    def close(self):
        if self.h:
            self.lib.ref_destroy(self.h)
            self.h = None

    def get(self):
        n = self.spec.nmol
        r, v, f = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros((n, 3))
        q, p, nn = np.zeros((n, 4)), np.zeros((n, 4)), np.zeros((n, 4))
        sc = np.zeros(14)
        self.lib.ref_get_state(self.h, _ptr(r), _ptr(v), _ptr(q), _ptr(p), _ptr(f), _ptr(nn),
                               _ptr(sc))
        return dict(r=r, v=v, q=q, p=p, f=f, n=nn, s=sc[0], Ps=sc[1], Q=sc[2], Pv=sc[3:6],
                    W=sc[6], L=sc[7:10], T=sc[10], P=sc[11], gkT=sc[12], H0=sc[13])

    def prop(self):
        o = np.zeros(21)
        self.lib.ref_get_property(self.h, _ptr(o))
        return dict(pot=o[0], lj=o[1], clmb=o[2], wall=o[3], vir=o[4:7], tra=o[7], rot=o[8],
                    kin=o[9], Tk=o[10], prs=o[11:15], tst=o[15], bst=o[16], tot=o[17],
                    ham=o[18], H0=o[19], gkT=o[20])

    def average(self):
        o = np.zeros(NUM_AVG)
        self.lib.ref_get_average(self.h, _ptr(o))
        return o

    def property_line(self):
        o = np.zeros(26)
        self.lib.ref_get_property_line(self.h, _ptr(o))
        return o

    def write_chk(self, path):
        self.lib.ref_write_chk(self.h, path.encode())

    def fwall(self):
        o = np.zeros(2 * self.spec.nfwall)
        self.lib.ref_get_fwall(self.h, _ptr(o))
        return o.reshape(-1, 2)

    def __getattr__(self, name):
        fn = getattr(self.__dict__["lib"], "ref_" + name)
        return lambda *a: fn(self.h, *a)


def reference_parallel_steps(refs, nsteps, nthreads):
    lib = refs[0].lib
    arr = (C.c_void_p * len(refs))(*[r.h.value for r in refs])
    lib.ref_execute_steps_parallel(arr, len(refs), nsteps, nthreads)
