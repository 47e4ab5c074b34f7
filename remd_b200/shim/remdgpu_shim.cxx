// remdgpu_shim.cxx -- REMDGPU (src/remdgpu.h:92-238) over libremd_b200.so.
// Compile with the reference's src/ on the include path, in place of
// src/remdgpu.cu:
//   g++ -O2 -DSWITCHING -DENABLE_GPU -I<remd>/src -I<this repo>/include \
//       -I<this repo>/remd_b200/shim -c remdgpu_shim.cxx
// and link with -L<this repo>/remd_b200/_lib -lremd_b200.
#include "remdgpu.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <sstream>

void REMDGPU::check(remd_status st, const char* what) {
  if (st != REMD_OK) {
    std::fprintf(stderr, "error: %s: %s\n", what, remd_last_error());
    std::exit(EXIT_FAILURE);
  }
}

// Molecules holds the molecule type normalised to reduced units
// (src/molecules.cxx:99-103); the C-ABI takes moltype.txt units.
static remd_system_desc describe(const Molecules* m) {
  remd_system_desc d{};
  const Parameter& p = m->param;
  const MolType& mt = m->mlist[0];
  d.nmol = m->nmol;
  d.nsite = (int)mt.a.size();
  for (int k = 0; k < d.nsite; k++) {
    for (int x = 0; x < 3; x++) d.site_r[k][x] = mt.a[k].r[x] * unit_length / 1e-10;
    d.site_mass[k] = mt.a[k].m * unit_mass / (1e-3 / Na);
    d.site_sigma[k] = mt.a[k].s * unit_length / 1e-10;
    d.site_eps[k] = mt.a[k].e * unit_energy / (1e3 / Na);
    d.site_charge[k] = mt.a[k].q * unit_coulomb / ele;
  }
  d.tconstant = p.tconstant;
  d.pconstant = p.pconstant;
  d.confined = p.confined;
  d.dt_fs = p.dt;
  d.rcut = p.rcut;
  d.rswitch = p.rswitch;
  d.nfwall = p.nfwall;
  d.wall_length = p.wall_length;
  d.sgm_wall = p.sgm_wall;
  d.eps_wall = p.eps_wall;
  d.rho_wall = p.rho_wall;
  d.interval = p.interval;
  return d;
}

REMDGPU::REMDGPU(Molecules** mlcls, const unsigned int nreplica) : nreplica_(nreplica) {
  const remd_system_desc d = describe(mlcls[0]);
  nmol_ = d.nmol;
  std::vector<remd_replica_init> init(nreplica);
  std::vector<std::vector<double>> keep;
  for (unsigned r = 0; r < nreplica; r++) {
    const Molecules* m = mlcls[r];
    std::vector<double> rr(3 * nmol_), v(3 * nmol_), q(4 * nmol_), p(4 * nmol_), mass(nmol_), I(3 * nmol_);
    for (int i = 0; i < nmol_; i++) {
      for (int x = 0; x < 3; x++) {
        rr[3 * i + x] = m->mlcl[i].r[x];
        v[3 * i + x] = m->mlcl[i].v[x];
        I[3 * i + x] = m->mlcl[i].i[x];
      }
      for (int x = 0; x < 4; x++) {
        q[4 * i + x] = m->mlcl[i].q[x];
        p[4 * i + x] = m->mlcl[i].p[x];
      }
      mass[i] = m->mlcl[i].m;
    }
    keep.push_back(rr); keep.push_back(v); keep.push_back(q);
    keep.push_back(p); keep.push_back(mass); keep.push_back(I);
    const size_t b = keep.size() - 6;
    remd_replica_init& ri = init[r];
    ri.r = keep[b].data(); ri.v = keep[b + 1].data(); ri.q = keep[b + 2].data();
    ri.p = keep[b + 3].data(); ri.mass = keep[b + 4].data(); ri.inertia = keep[b + 5].data();
    ri.s = m->tst->s; ri.Ps = m->tst->Ps; ri.Q = m->tst->Q;
    for (int x = 0; x < 3; x++) { ri.Pv[x] = m->bst->Pv[x]; ri.L[x] = m->L[x]; }
    ri.W = m->bst->W;
    ri.T = m->T;
    ri.P = m->P;
  }
  const int reps = (int)nreplica;
  check(remd_create(&d, 1, &reps, init.data(), REMD_PREC_FP32, mlcls[0]->param.gpu_offset, &h_),
        "remd_create");
  avg_.assign((size_t)nreplica * REMD_NUM_AVERAGES, 0.0);
  check(remd_get_all_averages(h_, avg_.data()), "remd_get_all_averages");
}

REMDGPU::~REMDGPU() { remd_destroy(h_); }

void REMDGPU::ExecuteSteps(double* T, double* P) {
  check(remd_execute_steps(h_, T, P), "remd_execute_steps");
  check(remd_get_all_averages(h_, avg_.data()), "remd_get_all_averages");
}

void REMDGPU::GetBackAllVariablesFromGPU() { check(remd_synchronize(h_), "remd_synchronize"); }

Average REMDGPU::GetAverages(unsigned int rep) {
  Average a;
  for (int k = 0; k < Average::NUM_ELEM && k < REMD_NUM_AVERAGES; k++)
    a.sum[k] = avg_[(size_t)rep * REMD_NUM_AVERAGES + k];
  return a;
}

float REMDGPU::GetPotential(unsigned int rep) {
  const double* a = &avg_[(size_t)rep * REMD_NUM_AVERAGES];
  return (float)(a[REMD_AVG_LJ] + a[REMD_AVG_CLMB] + a[REMD_AVG_WALL]);
}

float REMDGPU::GetVolume(unsigned int rep) { return (float)avg_[(size_t)rep * REMD_NUM_AVERAGES + REMD_AVG_VOL]; }

void REMDGPU::ConvertVariablesToHost(Molecules** mlcls) {
  std::vector<double> r(3 * nmol_), v(3 * nmol_), q(4 * nmol_), p(4 * nmol_), f(3 * nmol_), n(4 * nmol_);
  for (unsigned rep = 0; rep < nreplica_; rep++) {
    remd_state_view sv{};
    sv.r = r.data(); sv.v = v.data(); sv.q = q.data(); sv.p = p.data(); sv.f = f.data(); sv.n = n.data();
    check(remd_get_state(h_, (int)rep, &sv), "remd_get_state");
    Molecules* m = mlcls[rep];
    for (int i = 0; i < nmol_; i++) {
      for (int x = 0; x < 3; x++) {
        m->mlcl[i].r[x] = r[3 * i + x];
        m->mlcl[i].v[x] = v[3 * i + x];
        m->mlcl[i].f[x] = f[3 * i + x];
      }
      for (int x = 0; x < 4; x++) {
        m->mlcl[i].q[x] = q[4 * i + x];
        m->mlcl[i].p[x] = p[4 * i + x];
        m->mlcl[i].n[x] = n[4 * i + x];
      }
    }
    m->tst->s = sv.s;
    m->tst->Ps = sv.Ps;
    for (int x = 0; x < 3; x++) { m->bst->Pv[x] = sv.Pv[x]; m->L[x] = sv.L[x]; }
    m->prop.lj = sv.lj; m->prop.clmb = sv.clmb; m->prop.wall = sv.wall; m->prop.pot = sv.pot;
    for (int x = 0; x < 3; x++) m->prop.vir[x] = sv.vir[x];
    m->prop.H0 = sv.H0;
  }
}

void REMDGPU::OutputCheckPoint(const char* prefix, const int* index) {
  for (unsigned rep = 0; rep < nreplica_; rep++) {
    std::stringstream s;
    s << prefix << std::setw(4) << std::setfill('0') << (index ? index[rep] : (int)rep) << ".chk";
    check(remd_write_chk(h_, (int)rep, s.str().c_str()), "remd_write_chk");
  }
}

// .cdv snapshots of every replica (src/remdgpu.cu:700-804); the reference writes
// them per replica slot, not per condition, so index is not used there either.
void REMDGPU::OutputCDV(const char* prefix, const unsigned int step, const int* index) {
  (void)index;
  check(remd_output_cdv(h_, prefix, step), "remd_output_cdv");
}

void REMDGPU::PrintAll(std::ostream& os) {
  for (unsigned rep = 0; rep < nreplica_; rep++) {
    os << "replica " << rep;
    for (int k = 0; k < REMD_NUM_AVERAGES; k++) os << " " << avg_[(size_t)rep * REMD_NUM_AVERAGES + k];
    os << "\n";
  }
}

void REMDGPU::Diff(Molecules** mlcls, std::ostream& os) {
  std::vector<double> r(3 * nmol_);
  for (unsigned rep = 0; rep < nreplica_; rep++) {
    remd_state_view sv{};
    sv.r = r.data();
    check(remd_get_state(h_, (int)rep, &sv), "remd_get_state");
    double d = 0.0;
    for (int i = 0; i < nmol_; i++)
      for (int x = 0; x < 3; x++) d = std::fmax(d, std::fabs(r[3 * i + x] - mlcls[rep]->mlcl[i].r[x]));
    os << "replica " << rep << " max |dr| (box fraction) " << d << "\n";
  }
}
