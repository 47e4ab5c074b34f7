"""Shared helpers for the parity tests."""
import json
import os

import numpy as np

from remd_b200 import systems as S
from remd_b200.inputs import ReplicaState, SystemSpec, UNIT_PRESS, UNIT_TEMP, load_model

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = {
    "tip3p_bulk_npt": ("tip3p", 0, 1, 1, 64, 101),
    "tip4p_tube_npz": ("tip4p", 1, 2, 1, 96, 102),
    "tip5p_bulk_nvt": ("tip5p", 0, 0, 1, 64, 103),
    "tip4p_bulk_nve": ("tip4p", 0, 0, 0, 64, 104),
    "tip5p_tube_nvt": ("tip5p", 1, 0, 1, 80, 105),
    "tip3p_tube_npz": ("tip3p", 1, 2, 1, 72, 106),
    "tip4p_bulk_vscale": ("tip4p", 0, 0, 2, 64, 107),
    "tip3p_tube_npz_vscale": ("tip3p", 1, 2, 2, 72, 108),
    "tip4p_slit_nvt": ("tip4p", 2, 0, 1, 96, 109),
    "tip3p_slit_nve": ("tip3p", 2, 0, 0, 80, 110),
    "tip5p_slit_nvt": ("tip5p", 2, 0, 1, 72, 111),
}
NSTEPS = 20


def case_ensemble(name, interval=NSTEPS):
    model, confined, pcon, tcon, nmol, seed = CASES[name]
    return S.small_ensemble(model=model, confined=confined, nmol=nmol, ntemp=1, npress=1,
                            seed=seed, pconstant=pcon, tconstant=tcon, interval=interval)


def load_case(name):
    """Spec, initial state (from the committed fixture) and the reference outputs."""
    z = dict(np.load(os.path.join(GOLDEN, f"ref_{name}.npz")))
    ens = case_ensemble(name)
    sc = z["scal0"]
    st = ReplicaState(z["r0"], z["v0"], z["q0"], z["p0"], z["m"], z["I"], sc[0], sc[1], sc[2],
                      sc[3:6].copy(), sc[6], sc[7:10].copy(), sc[10], sc[11])
    return ens.spec, st, z


def golden_spec():
    """The reference's regression input (test/input/gpu.inp + gpu0000.chk)."""
    mt = load_model("tip4p")
    return SystemSpec(nmol=150, moltype=mt, tconstant=1, pconstant=2, confined=1, dt=2.0,
                      rcut=8.655, rswitch=6.655, nfwall=65536, wall_length=7.4, sgm_wall=3.277,
                      eps_wall=0.3886, rho_wall=0.38016, tstat_mass=0.5, bstat_mass=0.05,
                      interval=100)


def golden_line():
    return json.load(open(os.path.join(GOLDEN, "correct_line.json")))


def golden_conditions():
    return 200.0 / UNIT_TEMP, 4e9 / UNIT_PRESS


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


# (volume, potential) histogram pins: energy_min, energy_max (kJ/mol per molecule),
# volume_min, volume_max (A^3 per molecule), as in the .inp
HIST_RANGES = (-60.0, -20.0, 25.0, 35.0)


def histogram_samples(rng, nrep, nmol, nint):
    """Seeded per-interval Average rows and slot -> replica permutations; the
    potential and volume per molecule fall in [-41, -40) and [29.8, 30) so that
    the written histograms stay small (about 12 x 10 bins)."""
    out = []
    for _ in range(nint):
        avg = rng.normal(0.0, 1.0, (nrep, 19))
        avg[:, 0] = rng.uniform(-5.0, -4.9, nrep) * nmol
        avg[:, 1] = rng.uniform(-35.5, -35.0, nrep) * nmol
        avg[:, 2] = rng.uniform(-0.4, -0.1, nrep) * nmol
        avg[:, 3] = rng.uniform(29.8, 30.0, nrep) * nmol
        out.append((rng.permutation(nrep).astype(np.int32), avg))
    return out
