"""Host-side input model of the REMD engine: molecule types, .inp parameters,
.chk checkpoints and per-replica state, in the reference's layouts.

  moltype.txt  Molecules::MakeMolTypeList      src/molecules.cxx:69-131
  .inp         Parameter::read                 src/parameter.h:174-243
  .chk         IOManager::Read/WriteCheckPoint src/io_manager.cxx:528-634

State arrays use the reference's internal convention (what Molecules holds
after ReadCheckPoint): r is the box fraction in [0,1), v = v_real * L * s,
p = conjugate quaternion momentum * s; T and P are reduced.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

DATA_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")

# ---- reduced units, restated from src/unit.h:1-19 ----
NA = 6.0221367e+23
E0 = 8.8542e-12
ELE = 1.6021761e-19
KB = 1.3806488e-23
UNIT_MASS = 15.9994e-3 / NA
UNIT_LENGTH = 1.0e-10
UNIT_ENERGY = 1e3 / NA
UNIT_TIME = math.sqrt(UNIT_MASS * UNIT_LENGTH * UNIT_LENGTH / UNIT_ENERGY)
UNIT_COULOMB = math.sqrt(4. * math.pi * E0 * UNIT_ENERGY * UNIT_LENGTH)
UNIT_TEMP = UNIT_ENERGY / KB
UNIT_PRESS = UNIT_ENERGY / (UNIT_LENGTH ** 3)

MODEL_FILES = {"tip3p": "moltype_tip3p.txt", "tip4p": "moltype_tip4p.txt",
               "tip5p": "moltype_tip5p.txt"}


def moltype_path(model: str) -> str:
    return os.path.join(DATA_DIR, MODEL_FILES[model.lower()])


@dataclass
class MolType:
    """One molecule type as in moltype.txt (A, g/mol, A, kJ/mol, e)."""
    name: str
    names: list
    r: np.ndarray        # (nsite, 3) body-frame offsets from the centre of mass
    mass: np.ndarray
    sigma: np.ndarray
    eps: np.ndarray
    charge: np.ndarray

    @property
    def nsite(self):
        return len(self.mass)

    def reduced_mass(self) -> float:
        """Molecule mass in reduced units (MolType site masses summed)."""
        return float(np.sum(self.mass * (1e-3 / NA / UNIT_MASS)))

    def reduced_inertia(self) -> np.ndarray:
        """MolType::CalcIner (src/variables.h:316-334) in reduced units."""
        m = self.mass * (1e-3 / NA / UNIT_MASS)
        b = self.r * (1e-10 / UNIT_LENGTH)
        x, y, z = b[:, 0], b[:, 1], b[:, 2]
        return np.array([np.sum(m * (y * y + z * z)), np.sum(m * (z * z + x * x)),
                         np.sum(m * (x * x + y * y))])


def read_moltype(path) -> MolType:
    """First molecule block of a moltype file (src/molecules.cxx:69-131)."""
    with open(path) as f:
        lines = f.read().splitlines()
    i = 0
    while i < len(lines):
        tok = lines[i].split()
        i += 1
        if not tok or not tok[0][0].isalpha():
            continue
        n = int(tok[1])
        rows = [lines[i + k].split() for k in range(n)]
        return MolType(tok[0], [r[0] for r in rows],
                       np.array([[float(x) for x in r[1:4]] for r in rows]),
                       np.array([float(r[4]) for r in rows]),
                       np.array([float(r[5]) for r in rows]),
                       np.array([float(r[6]) for r in rows]),
                       np.array([float(r[7]) for r in rows]))
    raise ValueError(f"no molecule type in {path}")


def load_model(model: str) -> MolType:
    return read_moltype(moltype_path(model))


@dataclass
class SystemSpec:
    """The .inp parameters on the hot path (src/parameter.h:9-300)."""
    nmol: int
    moltype: MolType
    tconstant: int = 1
    pconstant: int = 0
    confined: int = 0
    dt: float = 2.0           # fs
    rcut: float = 10.0        # A
    rswitch: float = 8.0      # A
    nfwall: int = 0
    wall_length: float = 0.0  # A (tube radius or slit width)
    sgm_wall: float = 3.19
    eps_wall: float = 0.3135
    rho_wall: float = 0.3816
    tstat_mass: float = 1.0
    bstat_mass: float = 1.0
    interval: int = 100
    moltype_file: str = ""

    @property
    def mode(self) -> int:
        """Ensemble bit field, src/integrator.h:15-60 and src/molecules.h:168."""
        return (self.confined << 4) | (self.pconstant << 2) | self.tconstant

    def inp_text(self, moltype_path=None, interval=None, extra=""):
        mp = moltype_path or self.moltype_file
        d, b = os.path.split(os.path.abspath(mp))
        mt = self.moltype
        iv = self.interval if interval is None else interval
        return (f"input_prefix {d}/\nmtl_in {b}\nnmol {self.nmol}\n"
                f"natom {self.nmol * mt.nsite}\nnsite {mt.nsite}\ndt {self.dt!r}\n"
                f"rcut {self.rcut!r}\nrswitch {self.rswitch!r}\ntconstant {self.tconstant}\n"
                f"tstat_mass {self.tstat_mass!r}\npconstant {self.pconstant}\n"
                f"bstat_mass {self.bstat_mass!r}\ninterval {iv}\n"
                f"confined {self.confined}\nnfwall {self.nfwall}\n"
                f"wall_length {self.wall_length!r}\nsgm_wall {self.sgm_wall!r}\n"
                f"eps_wall {self.eps_wall!r}\nrho_wall {self.rho_wall!r}\n" + extra)


@dataclass
class ReplicaState:
    """Internal-unit state of one replica (as Molecules holds it after ReadCheckPoint)."""
    r: np.ndarray   # (n,3) box fraction
    v: np.ndarray   # (n,3) velocity * L * s
    q: np.ndarray   # (n,4)
    p: np.ndarray   # (n,4) conjugate momentum * s
    m: np.ndarray   # (n,)
    I: np.ndarray   # (n,3)
    s: float = 1.0
    Ps: float = 0.0
    Q: float = 1.0
    Pv: np.ndarray = field(default_factory=lambda: np.zeros(3))
    W: float = 1.0
    L: np.ndarray = field(default_factory=lambda: np.ones(3))
    T: float = 1.0   # reduced
    P: float = 0.0   # reduced

    @property
    def nmol(self):
        return len(self.m)

    def copy(self):
        return ReplicaState(self.r.copy(), self.v.copy(), self.q.copy(), self.p.copy(),
                            self.m.copy(), self.I.copy(), self.s, self.Ps, self.Q,
                            self.Pv.copy(), self.W, self.L.copy(), self.T, self.P)


def read_chk(path) -> ReplicaState:
    """Reader of the .chk layout (src/io_manager.cxx:528-591): nmol natom; per
    molecule r[A] v q[4] p m I[3] type id; s Ps Q; Pv[3] W; L[3]."""
    with open(path) as f:
        tok = f.read().split()
    nmol = int(tok[0])
    pos = 2
    rows = np.array(tok[pos:pos + 20 * nmol], dtype=float).reshape(nmol, 20)
    pos += 20 * nmol
    s, Ps, Q = (float(x) for x in tok[pos:pos + 3])
    pos += 3
    Pv = np.array(tok[pos:pos + 3], dtype=float)
    W = float(tok[pos + 3])
    pos += 4
    L = np.array(tok[pos:pos + 3], dtype=float)
    return ReplicaState(rows[:, 0:3] / L, rows[:, 3:6] * (L * s), rows[:, 6:10].copy(),
                        rows[:, 10:14] * s, rows[:, 14].copy(), rows[:, 15:18].copy(),
                        s, Ps, Q, Pv, W, L.copy())


def write_chk(path, st: ReplicaState, nsite: int):
    """Writer of the .chk layout (src/io_manager.cxx:593-634), without the trailing
    Property line."""
    L, s = st.L, st.s
    with open(path, "w") as f:
        f.write(f"{st.nmol} {st.nmol * nsite}\n")
        aid = 0
        for i in range(st.nmol):
            vals = list(st.r[i] * L) + list(st.v[i] / (L * s)) + list(st.q[i]) + \
                list(st.p[i] / s)
            f.write("".join(f" {x:e}" for x in vals))
            f.write(f" {st.m[i]:e} " + "".join(f" {x:e}" for x in st.I[i]))
            f.write(f" 0 {aid}\n")
            aid += nsite
        f.write(f"{s:e} {st.Ps:e} {st.Q:e}\n")
        f.write("".join(f" {x:e}" for x in st.Pv) + f" {st.W:e}\n")
        f.write("".join(f" {x:e}" for x in L) + "\n")
