"""Regenerate the committed golden fixtures from the reference itself.

Run in a container that has the reference sources (it builds oracle/_ref from
them with oracle/Makefile):

    python tests/golden/make_golden.py [case ...]     (all cases when none is named)
    python tests/golden/make_golden.py histograms     (ref_histograms.json only)

Writes, next to this script:
  gpu0000.chk          copy of the reference's test input (test/input/gpu0000.chk)
  correct_line.json    the reference's golden interval-0 line (test/correct:4)
  ref_histograms.json  the reference REMDInfo's histogram files for seeded samples
  ref_<case>.npz       for small seeded systems: the initial state and the
                       reference's own outputs (compiled reference CPU code,
                       generic FP64 build) after InitializeProperty (a force
                       snapshot) and after 20 MD steps.  Slit systems
                       (confined=2) use the build whose broken CPU slit wall
                       is replaced by the reference GPU kernel's lookup
                       (oracle/ref_slit_wall.cxx); everything else there is
                       the reference's own code.
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
    "tip4p_slit_nvt": ("tip4p", 2, 0, 1, 96, 109),
    "tip3p_slit_nve": ("tip3p", 2, 0, 0, 80, 110),
    "tip5p_slit_nvt": ("tip5p", 2, 0, 1, 72, 111),
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


def histograms(path):
    """ref_histograms.json: the reference REMDInfo's OutputHistogram files
    (src/remdinfo.cxx:723-758) after REMD::IncrementHistogram-style feeding
    (src/remd.cxx:803-813) of seeded samples (tests.common.histogram_samples)."""
    import tempfile
    from tests.common import HIST_RANGES, histogram_samples
    seed, nt, npr, nmol, nint = 9, 3, 2, 50, 40
    nrep = nt * npr
    lib = O._ref_lib()
    with tempfile.TemporaryDirectory() as tmp:
        inp = ("nmol %d\nntemp %d\nnpress %d\nnreplica %d\ntemp_min 250\ntemp_max 350\n"
               "press_min 1e5\npress_max 2e8\npconstant 1\nconfined 0\ntconstant 1\n"
               "energy_min %r\nenergy_max %r\nvolume_min %r\nvolume_max %r\n"
               "output_prefix %s\ninput_prefix %s\n" % ((nmol, nt, npr, nrep) + HIST_RANGES + (tmp, tmp)))
        h = lib.ref_remdinfo_create(inp.encode())
        Tc, Pc = np.linspace(2.0, 3.0, nrep), np.linspace(0.01, 0.1, nrep)
        for idx, avg in histogram_samples(np.random.default_rng(seed), nrep, nmol, nint):
            T, P = np.zeros(nrep), np.zeros(nrep)
            T[idx], P[idx] = Tc, Pc
            lib.ref_remdinfo_set_arrays(h, O._ptr(idx, O._ip), O._ptr(T), O._ptr(P))
            pot = np.ascontiguousarray(avg[:, 0] + avg[:, 1] + avg[:, 2])
            vol = np.ascontiguousarray(avg[:, 3])
            lib.ref_remdinfo_increment_histogram(h, O._ptr(pot), O._ptr(vol),
                                                 O._ptr(np.ascontiguousarray(avg)))
        lib.ref_remdinfo_output_histogram(h)
        files = [open(O.Histograms.file_name(tmp, Pc[c], Tc[c])).read() for c in range(nrep)]
    json.dump({"source": "REMDInfo::OutputHistogram (src/remdinfo.cxx:723-758)", "seed": seed,
               "nrep": nrep, "nmol": nmol, "nint": nint, "ranges": list(HIST_RANGES),
               "files": files}, open(path, "w"), indent=0)


def main():
    O.build_oracle()
    if sys.argv[1:] == ["histograms"]:
        histograms(os.path.join(HERE, "ref_histograms.json"))
        return
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
        # slit systems: the build whose CPU slit wall is the reference GPU kernel's
        # (oracle/ref_slit_wall.cxx); the reference's own CPU slit branch is broken
        variant = "slitwall" if spec.confined == 2 else "generic"
        ref = O.Reference(spec, st, spec.moltype_file, variant=variant)
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
