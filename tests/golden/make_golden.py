"""Regenerate the committed golden fixtures from the reference itself.

Run in a container that has the reference sources (it builds oracle/_ref from
them with oracle/Makefile):

    python tests/golden/make_golden.py [case ...]     (all cases when none is named)

Writes, next to this script:
  gpu0000.chk          copy of the reference's test input (test/input/gpu0000.chk)
  correct_line.json    the reference's golden interval-0 line (test/correct:4)
  ref_<case>.npz       for small seeded systems: the initial state and the
                       reference's own outputs (compiled reference CPU code,
                       generic FP64 build) after InitializeProperty (a force
                       snapshot) and after 20 MD steps.
The tests compare the C oracle, and through it the CUDA engine, with these.
"""
import json
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from remd_b200 import systems as S  # noqa: E402

REF = os.environ.get("REMD_REFERENCE", "/root/reference")

# name -> (model, confined, pconstant, tconstant, nmol, seed)
CASES = {
    "tip3p_bulk_npt": ("tip3p", 0, 1, 1, 64, 101),
    "tip4p_tube_npz": ("tip4p", 1, 2, 1, 96, 102),
    "tip5p_bulk_nvt": ("tip5p", 0, 0, 1, 64, 103),
    "tip4p_bulk_nve": ("tip4p", 0, 0, 0, 64, 104),
    "tip5p_tube_nvt": ("tip5p", 1, 0, 1, 80, 105),
    "tip3p_tube_npz": ("tip3p", 1, 2, 1, 72, 106),
    "tip4p_bulk_vscale": ("tip4p", 0, 0, 2, 64, 107),
    "tip3p_tube_npz_vscale": ("tip3p", 1, 2, 2, 72, 108),
}
NSTEPS = 20


def case_ensemble(name):
    model, confined, pcon, tcon, nmol, seed = CASES[name]
    return S.small_ensemble(model=model, confined=confined, nmol=nmol, ntemp=1, npress=1,
                            seed=seed, pconstant=pcon, tconstant=tcon, interval=NSTEPS)


def ref_outputs(ref, spec):
    g = ref.get()
    pr = ref.prop()
    wall = pr["wall"] if spec.confined else 0.0   # Property::wall is uninitialised for bulk
    return dict(f=g["f"], n=g["n"], r=g["r"], v=g["v"], q=g["q"], p=g["p"],
                scal=np.array([g["s"], g["Ps"], *g["Pv"], *g["L"], g["H0"]]),
                ener=np.array([pr["lj"], pr["clmb"], wall, *pr["vir"], pr["tra"], pr["rot"],
                               pr["tot"] - pr["wall"] + wall]))


def main():
    O.build_oracle()
    shutil.copy(os.path.join(REF, "test/input/gpu0000.chk"), os.path.join(HERE, "gpu0000.chk"))
    with open(os.path.join(REF, "test/correct")) as f:
        line = f.read().splitlines()[3].split()
    cols = ["pot", "vol", "T_red", "Pz_red", "rot", "tra", "s", "Ps", "Pv_z", "drift"]
    json.dump({"source": "test/correct:4", "columns": cols,
               "values": [float(x) for x in line[3:]]},
              open(os.path.join(HERE, "correct_line.json"), "w"), indent=1)
    for name in (sys.argv[1:] or CASES):
        ens = case_ensemble(name)
        spec, st = ens.spec, ens.states[0]
        ref = O.Reference(spec, st, spec.moltype_file)
        ref.initialize_property()
        snap = ref_outputs(ref, spec)
        ref.execute_steps(NSTEPS)
        after = ref_outputs(ref, spec)
        avg = ref.average()
        np.savez_compressed(
            os.path.join(HERE, f"ref_{name}.npz"),
            r0=st.r, v0=st.v, q0=st.q, p0=st.p, m=st.m, I=st.I,
            scal0=np.array([st.s, st.Ps, st.Q, *st.Pv, st.W, *st.L, st.T, st.P]),
            **{f"snap_{k}": v for k, v in snap.items()},
            **{f"after_{k}": v for k, v in after.items()}, avg=avg)
        ref.close()
        print("wrote", name)


if __name__ == "__main__":
    main()
