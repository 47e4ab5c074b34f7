// io_manager_harness.cxx -- the IOManager members that the reference's REMD
// driver (src/remd.cxx, src/main.cxx) calls, written here so that the driver
// itself compiles unmodified and runs on the engine through the REMDGPU shim.
// The reference's own src/io_manager.cxx cannot be compiled: it includes the
// VMD molfile plugin sources (gromacsplugin.C), which are not vendored.
//
// TEST INFRASTRUCTURE ONLY (oracle/Makefile -> oracle/_ref/remd_driver).  It
// covers what a GPU run of the driver uses: .chk input (ReadInputs), .chk and
// .gro output (UpdateOutputs).  .gro/.trr/.xyz/.cdv inputs are rejected; the
// GPU path writes .cdv snapshots through REMDGPU::OutputCDV, not WriteCDV.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "io_manager.h"
#include "remd_b200.h"

// File names as InputParam(const Parameter) forms them (src/io_manager.cxx:88-156):
// prefix + name + extension, "null" kept as is; the checkpoint output name has
// no extension here (WriteCheckPoint appends the replica index and ".chk").
InputParam::InputParam(const Parameter param) {
  nmol = param.nmol;
  natom = param.natom;
  auto name = [](char* dst, const std::string& v, const std::string& pfx, const char* ext) {
    const std::string s = (v == "null") ? v : pfx + v + ext;
    std::snprintf(dst, 256, "%s", s.c_str());
  };
  name(igro, param.gro_in, param.input_prefix, ".gro");
  name(itrr, param.trr_in, param.input_prefix, ".trr");
  name(ichk, param.chk_in, param.input_prefix, ".chk");
  name(itkw, param.tkw_in, param.input_prefix, ".tkw");
  name(ixyz, param.xyz_in, param.input_prefix, ".xyz");
  name(icdv, param.cdv_in, param.input_prefix, ".cdv");
  name(ogro, param.gro_out, param.output_prefix, ".gro");
  name(otrr, param.trr_out, param.output_prefix, ".trr");
  name(ochk, param.chk_out, param.output_prefix, "");
  name(oene, param.ene_out, param.output_prefix, ".ene");
  name(ocdv, param.cdv_out, param.output_prefix, "");
}

IOManager::IOManager(const Parameter p) {
  iprm = new InputParam(p);
  nmol = p.nmol;
  natom = p.natom;
  atom = nullptr;
  rg = nullptr;
  rt = wt = nullptr;
}

IOManager::~IOManager() { delete iprm; }

// ReadCheckPoint (src/io_manager.cxx:528-591) through the engine's .chk reader,
// which converts the state the same way (r / L, v * L s, p * s).
void IOManager::ReadInputs(Molecule* m, Thermostat* tst, Barostat* bst, MolTypeList ml, const int n,
                           const int na, dvec3& L, Property& prop) {
  (void)na;
  (void)prop;
  if (std::string(iprm->ichk) == "null") {
    std::fprintf(stderr, "io_manager_harness: only .chk input is supported\n");
    std::exit(EXIT_FAILURE);
  }
  std::vector<double> r(3 * n), v(3 * n), q(4 * n), p(4 * n), mass(n), I(3 * n), sc(10);
  if (remd_read_chk(iprm->ichk, n, r.data(), v.data(), q.data(), p.data(), mass.data(), I.data(),
                    sc.data()) != REMD_OK) {
    std::fprintf(stderr, "io_manager_harness: %s\n", remd_last_error());
    std::exit(EXIT_FAILURE);
  }
  int atom_count = 0;
  for (int i = 0; i < n; i++) {
    for (int x = 0; x < 3; x++) {
      m[i].r[x] = r[3 * i + x];
      m[i].v[x] = v[3 * i + x];
      m[i].i[x] = I[3 * i + x];
    }
    for (int x = 0; x < 4; x++) {
      m[i].q[x] = q[4 * i + x];
      m[i].p[x] = p[4 * i + x];
    }
    m[i].m = mass[i];
    m[i].type = 0;
    m[i].id = atom_count;
    atom_count += (int)ml[0].a.size();
  }
  tst->s = sc[0];
  tst->Ps = sc[1];
  tst->Q = sc[2];
  for (int x = 0; x < 3; x++) {
    bst->Pv[x] = sc[3 + x];
    L[x] = sc[7 + x];
  }
  bst->W = sc[6];
}

// WriteCheckPoint (src/io_manager.cxx:593-634) through the engine's .chk writer
// (remd_write_chk_arrays), with the caller's Property on the last line.
void IOManager::WriteCheckPoint(const Molecule* m, const Thermostat* tst, const Barostat* bst,
                                const dvec3 L, const Property prop, const int index) {
  char path[300];
  std::snprintf(path, sizeof(path), "%s%04d.chk", iprm->ochk, index);
  std::vector<double> r(3 * nmol), v(3 * nmol), q(4 * nmol), p(4 * nmol);
  for (int i = 0; i < nmol; i++) {
    for (int x = 0; x < 3; x++) { r[3 * i + x] = m[i].r[x]; v[3 * i + x] = m[i].v[x]; }
    for (int x = 0; x < 4; x++) { q[4 * i + x] = m[i].q[x]; p[4 * i + x] = m[i].p[x]; }
  }
  const double I[3] = {m[0].i[0], m[0].i[1], m[0].i[2]};
  const double scal[10] = {tst->s, tst->Ps, tst->Q, bst->Pv[0], bst->Pv[1], bst->Pv[2], bst->W,
                           L[0], L[1], L[2]};
  const int nsite = natom / nmol;
  // the caller's Property, as the reference's operator<< prints it (src/variables.h:51-74)
  const double nave = (prop.nave != 0) ? (double)prop.nave : 1.0;
  const double pv[26] = {
      prop.time, prop.pot, prop.tra, prop.rot, prop.kin, prop.tsm, prop.tsp, prop.tst, prop.bst,
      prop.tot, prop.ham, prop.tmo[0], prop.tmo[1], prop.tmo[2], prop.Tave / nave,
      prop.prs[0], prop.prs[1], prop.prs[2], prop.prs[3], prop.vir[0], prop.vir[1], prop.vir[2],
      prop.Pave[0] / nave, prop.Pave[1] / nave, prop.Pave[2] / nave, prop.Pave[3] / nave};
  if (remd_write_chk_arrays(path, nmol, nsite, r.data(), v.data(), q.data(), p.data(), m[0].m, I, scal,
                            pv) != REMD_OK) {
    std::fprintf(stderr, "io_manager_harness: %s\n", remd_last_error());
    std::exit(EXIT_FAILURE);
  }
}

// UpdateOutputs (src/io_manager.cxx:636-651): .gro (sites r L + R(q) b in nm,
// velocities 0, box in nm, the reference's write_gro_file) and .chk.
void IOManager::UpdateOutputs(const Molecule* m, const Thermostat* tst, const Barostat* bst,
                              const Property prop, const dvec3 L, MolTypeList ml, const int index) {
  if (std::string(iprm->ogro) != "null") {
    std::vector<AtomGro> a(natom);
    int k = 0;
    for (int i = 0; i < nmol; i++) {
      const MolType& mt = ml[m[i].type];
      for (unsigned j = 0; j < mt.a.size(); j++, k++) {
        std::snprintf(a[k].MolName, sizeof(a[k].MolName), "%s", mt.name.c_str());
        std::snprintf(a[k].AtomName, sizeof(a[k].AtomName), "%s", mt.a[j].name.c_str());
        a[k].MolID = i + 1;
        a[k].AtomID = k + 1;
        const dvec3 site = body_to_space(m[i].q, mt.a[j].r);
        for (int d = 0; d < 3; d++) {
          a[k].coor[d] = (m[i].r[d] * L[d] + site[d]) * 0.1;
          a[k].vel[d] = 0.0;
        }
      }
    }
    dvec3 box;
    for (int d = 0; d < 3; d++) box[d] = L[d] * 0.1;
    char comment[8] = "test";
    write_gro_file(iprm->ogro, natom, a.data(), box, comment);
  }
  if (std::string(iprm->ochk) != "null") WriteCheckPoint(m, tst, bst, L, prop, index);
}

void IOManager::WriteCDV(const Molecule*, const MolTypeList, const dvec3, const long) {
  std::fprintf(stderr, "io_manager_harness: WriteCDV is the CPU path's; the GPU path writes .cdv "
                       "through REMDGPU::OutputCDV\n");
}
