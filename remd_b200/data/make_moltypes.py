"""Write moltype_tip3p.txt / moltype_tip4p.txt / moltype_tip5p.txt.

The files use the reference's moltype.txt layout (read by
Molecules::MakeMolTypeList, src/molecules.cxx:69-131): a "Name natom" line,
then one line per site "AtomName x y z mass sigma epsilon charge" in
A, g/mol, A, kJ/mol, e.  Site coordinates are in the principal body frame,
centred on the centre of mass: x along the H-O-H bisector (pointing from the
hydrogens to the oxygen), y in the molecular plane, z normal to it.

Geometry and parameters are the published ones:
  TIP3P  Jorgensen et al., J. Chem. Phys. 79, 926 (1983)
  TIP4P  Jorgensen et al., J. Chem. Phys. 79, 926 (1983)
  TIP5P  Mahoney & Jorgensen, J. Chem. Phys. 112, 8910 (2000)
Oxygen is always site 0 (the only Lennard-Jones site); charged sites follow.
"""
import math
import os

M_O, M_H = 15.9994, 1.008
R_OH, HOH = 0.9572, 104.52


def _water(extra):
    half = math.radians(HOH / 2.0)
    # O at origin, H's toward -x
    sites = [("OW", [0.0, 0.0, 0.0], M_O),
             ("HW1", [-R_OH * math.cos(half), R_OH * math.sin(half), 0.0], M_H),
             ("HW2", [-R_OH * math.cos(half), -R_OH * math.sin(half), 0.0], M_H)]
    sites += extra
    mtot = sum(m for _, _, m in sites)
    com = [sum(r[d] * m for _, r, m in sites) / mtot for d in range(3)]
    return [(n, [r[d] - com[d] for d in range(3)], m) for n, r, m in sites]


def models():
    tip3p = _water([])
    tip4p = _water([("MW", [-0.15, 0.0, 0.0], 0.0)])
    lh = math.radians(109.47 / 2.0)
    tip5p = _water([("LP1", [0.70 * math.cos(lh), 0.0, 0.70 * math.sin(lh)], 0.0),
                    ("LP2", [0.70 * math.cos(lh), 0.0, -0.70 * math.sin(lh)], 0.0)])
    return {
        "TIP3P": (tip3p, [3.15061, 0.0, 0.0], [0.6364, 0.0, 0.0], [-0.834, 0.417, 0.417]),
        "TIP4P": (tip4p, [3.15365, 0, 0, 0], [0.6485, 0, 0, 0], [0.0, 0.52, 0.52, -1.04]),
        "TIP5P": (tip5p, [3.12, 0, 0, 0, 0], [0.6694, 0, 0, 0, 0], [0.0, 0.241, 0.241, -0.241, -0.241]),
    }


def write_all(outdir):
    for name, (sites, sig, eps, q) in models().items():
        lines = ["#MolName natom",
                 "#AtomName r.x r.y r.z mass sigma epsilon charge",
                 "#angstrom x 3, g/mol, angstrom, kJ/mol, e",
                 f" {name} {len(sites)}"]
        for k, (an, r, m) in enumerate(sites):
            lines.append(f" {an:>5s} {r[0]: .7e} {r[1]: .7e} {r[2]: .7e} {m: .5e} "
                         f"{sig[k]: .5e} {eps[k]: .6e} {q[k]: .4e}")
        with open(os.path.join(outdir, f"moltype_{name.lower()}.txt"), "w") as f:
            f.write("\n".join(lines) + "\n")


if __name__ == "__main__":
    write_all(os.path.dirname(os.path.abspath(__file__)))
