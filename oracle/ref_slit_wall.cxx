// ref_slit_wall.cxx -- ForceCalculator::Confined for the "slit wall" build of
// the reference's CPU objects (oracle/_ref/libremdref_slitwall.so).
// TEST INFRASTRUCTURE ONLY: the engine never links it.
//
// The reference's CPU slit branch is broken (src/force_calculator.cxx:1556-1561:
// it interpolates at the absolute z instead of the distance from the mid-plane,
// multiplies by the z of another atom, adds nothing to the energy nor to the
// molecule force), and its tuned branch asserts (1525).  The reference's GPU
// kernel is the only correct slit wall it has (src/remdgpu.cu:1708-1720): the
// oxygen site's distance |z| from the slit mid-plane indexes the same table
// ForceCalculator::CalcWallForce builds (src/force_calculator.cxx:163-199) at
// half its CPU spacing (tex1D at 2|z|/R over nfwall entries), the force acts
// along sign(z) and the energy goes to the wall term.
//
// oracle/Makefile compiles the reference's force_calculator.cxx with
// -DConfined=ConfinedCpuReference, so that the reference's own Molecules /
// integrator / Switching code calls this function instead.  Everything else
// the reference executes is its own code, unmodified: Switching,
// ConvertToAtoms / ConvertFromAtoms, D1-D6, CalcProperties and the wall table.
// This build pins the engine's slit physics to executed reference code except
// for the lookup below, a restatement of the GPU kernel's.
//
// The tube branch is the reference CPU's generic branch
// (src/force_calculator.cxx:1544-1555) with its base index clamped to
// nfwall-2, as the engine and remd_oracle.c clamp it (the reference reads one
// entry past the table there).
#include "molecules.h"   // Molecule, Atom, MolTypeList, ForceCalculator

#include <cmath>

void ForceCalculator::Confined(Molecule* m, Atom* a, const MolTypeList mtl, const dvec3 L,
                               const int nmol, Property& prop, const int*, const int*) {
  const double dr = wall_length / (double)nfwall;
  int a_count = 0;
  prop.wall = 0.0;
  for (int i = 0; i < nmol; i++) {
    for (unsigned int ii = 0; ii < mtl[m[i].type].a.size(); ii++) {
      if (a[a_count].t == 0) {   // oxygen site only
        if (confined_dim == 1) {
          dvec3 r_i = a[a_count].r - L * 0.5;
          const double r01 = sqrt(r_i[0] * r_i[0] + r_i[1] * r_i[1]);
          int index = (int)(r01 / dr);
          if (index > nfwall - 2) index = nfwall - 2;
          const double f = (fwall[index + 1][0] - fwall[index][0]) / dr * (r01 - dr * index) + fwall[index][0];
          const double e = (fwall[index + 1][1] - fwall[index][1]) / dr * (r01 - dr * index) + fwall[index][1];
          a[a_count].f[0] += f * r_i[0];
          a[a_count].f[1] += f * r_i[1];
          m[i].f[0] += f * r_i[0];
          m[i].f[1] += f * r_i[1];
          a[a_count].e += e;
          prop.wall += e;
        } else if (confined_dim == 2) {
          const double z = a[a_count].r[2] - 0.5 * L[2];
          const double za = std::fabs(z);
          const double dir = (za != 0.0) ? z / za : 1.0;
          const double hdr = 0.5 * dr;   // the GPU texture's spacing: R / (2 nfwall)
          int index = (int)(za / hdr);
          if (index > nfwall - 2) index = nfwall - 2;
          const double f = (fwall[index + 1][0] - fwall[index][0]) / hdr * (za - hdr * index) + fwall[index][0];
          const double e = (fwall[index + 1][1] - fwall[index][1]) / hdr * (za - hdr * index) + fwall[index][1];
          a[a_count].f[2] += f * dir;
          m[i].f[2] += f * dir;
          a[a_count].e += e;
          prop.wall += e;
        }
      }
      a_count++;
    }
  }
}
