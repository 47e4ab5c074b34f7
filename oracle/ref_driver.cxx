// ref_driver.cxx -- a C-ABI around the reference's own CPU objects
// (Molecules, ForceCalculator, integrator, REMDInfo), compiled unmodified from
// the reference's src/ by oracle/Makefile into oracle/_ref/libremdref*.so.
//
// TEST INFRASTRUCTURE ONLY: it pins the C restatement (remd_oracle.c) and is
// the timed CPU baseline in bench.py.  The engine never links it.
//
// The reference's .chk reader (src/io_manager.cxx:528-591) cannot be compiled
// (it needs the unvendored VMD molfile plugin), so the caller passes the state
// arrays already converted the way ReadCheckPoint converts them: r as a box
// fraction, v scaled by L*s, p scaled by s.
#include "gro.h"
#include "molecules.h"
#include "remdinfo.h"

#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

namespace {
struct RefHandle {
  Parameter param;
  Molecules* m = nullptr;
};
}  // namespace

extern "C" {

void* ref_create(const char* inp_text) {
  auto* h = new RefHandle;
  std::istringstream is(inp_text);
  h->param.read(is);
  h->m = new Molecules(h->param);
  return h;
}

// ForceCalculator's destructor frees `fwall` even when it was never allocated
// (bulk systems, src/force_calculator.cxx:54-110), so a Molecules object is
// deliberately leaked rather than deleted.
void ref_destroy(void* hp) { (void)hp; }

int ref_natom(void* hp) { return static_cast<RefHandle*>(hp)->m->natom; }

void ref_set_state(void* hp, const double* r, const double* v, const double* q,
                   const double* p, const double* mass, const double* I, double s,
                   double Ps, double Q, const double* Pv, double W, const double* L) {
  Molecules* m = static_cast<RefHandle*>(hp)->m;
  int id = 0;
  for (int i = 0; i < m->nmol; i++) {
    Molecule& a = m->mlcl[i];
    for (int d = 0; d < 3; d++) {
      a.r[d] = r[3 * i + d];
      a.v[d] = v[3 * i + d];
      a.i[d] = I[3 * i + d];
    }
    for (int d = 0; d < 4; d++) {
      a.q[d] = q[4 * i + d];
      a.p[d] = p[4 * i + d];
    }
    a.m = mass[i];
    a.type = 0;
    a.id = id;
    id += m->mlist[0].a.size();
  }
  m->tst->s = s;
  m->tst->Ps = Ps;
  m->tst->Q = Q;
  for (int d = 0; d < 3; d++) {
    m->bst->Pv[d] = Pv[d];
    m->L[d] = L[d];
  }
  m->bst->W = W;
}

// scal: s Ps Q Pv0 Pv1 Pv2 W L0 L1 L2 T P gkT H0
void ref_get_state(void* hp, double* r, double* v, double* q, double* p, double* f,
                   double* n, double* scal) {
  Molecules* m = static_cast<RefHandle*>(hp)->m;
  for (int i = 0; i < m->nmol; i++) {
    const Molecule& a = m->mlcl[i];
    for (int d = 0; d < 3; d++) {
      if (r) r[3 * i + d] = a.r[d];
      if (v) v[3 * i + d] = a.v[d];
      if (f) f[3 * i + d] = a.f[d];
    }
    for (int d = 0; d < 4; d++) {
      if (q) q[4 * i + d] = a.q[d];
      if (p) p[4 * i + d] = a.p[d];
      if (n) n[4 * i + d] = a.n[d];
    }
  }
  if (scal) {
    scal[0] = m->tst->s;
    scal[1] = m->tst->Ps;
    scal[2] = m->tst->Q;
    for (int d = 0; d < 3; d++) scal[3 + d] = m->bst->Pv[d];
    scal[6] = m->bst->W;
    for (int d = 0; d < 3; d++) scal[7 + d] = m->L[d];
    scal[10] = m->T;
    scal[11] = m->P;
    scal[12] = m->prop.gkT;
    scal[13] = m->prop.H0;
  }
}

// out: pot lj clmb wall vir0 vir1 vir2 tra rot kin T prs0 prs1 prs2 prs3 tst bst tot ham H0 gkT
void ref_get_property(void* hp, double* out) {
  const Property& pr = static_cast<RefHandle*>(hp)->m->prop;
  const double vals[] = {pr.pot,   pr.lj,     pr.clmb,   pr.wall,   pr.vir[0], pr.vir[1], pr.vir[2],
                         pr.tra,   pr.rot,    pr.kin,    pr.T,      pr.prs[0], pr.prs[1], pr.prs[2],
                         pr.prs[3], pr.tst,   pr.bst,    pr.tot,    pr.ham,    pr.H0,     pr.gkT};
  std::memcpy(out, vals, sizeof(vals));
}

// The 26 numbers of the .chk Property line, in operator<< order (src/variables.h:51-74).
void ref_get_property_line(void* hp, double* out) {
  const Property& p = static_cast<RefHandle*>(hp)->m->prop;
  const double nave = (p.nave != 0) ? (double)p.nave : 1.0;
  const double v[26] = {p.time, p.pot, p.tra, p.rot, p.kin, p.tsm, p.tsp, p.tst, p.bst, p.tot, p.ham,
                        p.tmo[0], p.tmo[1], p.tmo[2], p.nave != 0 ? p.Tave / nave : p.Tave,
                        p.prs[0], p.prs[1], p.prs[2], p.prs[3], p.vir[0], p.vir[1], p.vir[2],
                        p.Pave[0] / nave, p.Pave[1] / nave, p.Pave[2] / nave, p.Pave[3] / nave};
  std::memcpy(out, v, sizeof(v));
}

// A .chk of the object's state written with the stream statements of
// IOManager::WriteCheckPoint (src/io_manager.cxx:611-632) and the reference's
// own operator<< for Vector (src/vector.h:141-147) and Property
// (src/variables.h:51-74).  io_manager.cxx itself cannot be compiled here.
void ref_write_chk(void* hp, const char* path) {
  Molecules* m = static_cast<RefHandle*>(hp)->m;
  std::ofstream ofs(path, std::ios_base::out);
  ofs << m->nmol << " " << m->natom << std::endl;
  for (int i = 0; i < m->nmol; i++) {
    const Molecule& a = m->mlcl[i];
    ofs << a.r * m->L;
    ofs << a.v / (m->L * m->tst->s);
    ofs << a.q;
    ofs << a.p / m->tst->s;
    ofs << " " << a.m;
    ofs << " " << a.i;
    ofs << " " << a.type;
    ofs << " " << a.id;
    ofs << std::endl;
  }
  ofs << m->tst->s << " " << m->tst->Ps << " " << m->tst->Q << std::endl;
  ofs << m->bst->Pv << " " << m->bst->W << std::endl;
  ofs << m->L << std::endl;
  ofs << m->prop << std::endl;
}

void ref_get_average(void* hp, double* out) {
  Average a = static_cast<RefHandle*>(hp)->m->GetAverage();
  for (int i = 0; i < Average::NUM_ELEM; i++) out[i] = a.sum[i];
}

void ref_get_fwall(void* hp, double* out) {
  Molecules* m = static_cast<RefHandle*>(hp)->m;
  for (int i = 0; i < m->fclcltr->nfwall; i++) {
    out[2 * i] = m->fclcltr->fwall[i][0];
    out[2 * i + 1] = m->fclcltr->fwall[i][1];
  }
}

void ref_set_temperature(void* hp, double T) { static_cast<RefHandle*>(hp)->m->SetTemperature(T); }
void ref_set_pressure(void* hp, double P) { static_cast<RefHandle*>(hp)->m->SetPressure(P); }
void ref_set_tstat_mass(void* hp, double Q) {
  Molecules* m = static_cast<RefHandle*>(hp)->m;
  m->tst->Q = Q;
  m->tst->flush();
}
void ref_initialize_property(void* hp) { static_cast<RefHandle*>(hp)->m->InitializeProperty(); }
void ref_calc_force(void* hp) { static_cast<RefHandle*>(hp)->m->CalcForcePot(); }
void ref_calc_properties(void* hp) { static_cast<RefHandle*>(hp)->m->CalcProperties(); }
void ref_update_hamiltonian(void* hp) { static_cast<RefHandle*>(hp)->m->UpdateHamiltonian(); }
void ref_velocity_scaling(void* hp) { static_cast<RefHandle*>(hp)->m->VelocityScaling(); }
void ref_ang_velocity_scaling(void* hp) { static_cast<RefHandle*>(hp)->m->AngVelocityScaling(); }
void ref_kill_momentum(void* hp) { static_cast<RefHandle*>(hp)->m->KillMomentum(); }
void ref_change_temperature(void* hp, double T) { static_cast<RefHandle*>(hp)->m->ChangeTemperature(T); }

// Molecules::ExecuteSteps runs param.interval steps then CalcProperties.
void ref_execute_steps(void* hp, int nsteps) {
  Molecules* m = static_cast<RefHandle*>(hp)->m;
  m->param.interval = nsteps;
  m->ExecuteSteps();
}

// Replica-parallel form: every handle advances nsteps on its own thread, the
// strongest CPU form of the reference (one replica per core).
void ref_execute_steps_parallel(void** hs, int nrep, int nsteps, int nthreads) {
  if (nthreads < 1) nthreads = 1;
  std::vector<std::thread> pool;
  for (int t = 0; t < nthreads; t++) {
    pool.emplace_back([=]() {
      for (int r = t; r < nrep; r += nthreads) ref_execute_steps(hs[r], nsteps);
    });
  }
  for (auto& th : pool) th.join();
}

// ---- exchange on top of the reference's compiled REMDInfo ----
// REMD::ReplicaExchange (src/remd.cxx:486-538) restated with an injected
// uniform stream in place of rand()/RAND_MAX.
void* ref_remdinfo_create(const char* inp_text) {
  Parameter p;
  std::istringstream is(inp_text);
  p.read(is);
  return new REMDInfo(p);
}
// REMDInfo's destructor frees its Histogram objects with delete[] on memory
// from new (src/remdinfo.cxx:296-300), so the handle is deliberately leaked.
void ref_remdinfo_destroy(void*) {}
void ref_remdinfo_arrays(void* h, int* index, double* T, double* P) {
  REMDInfo* ri = static_cast<REMDInfo*>(h);
  for (int i = 0; i < ri->GetNumReplica(); i++) {
    if (index) index[i] = ri->GetIndex(i);
    if (T) T[i] = ri->GetTemperature(i);
    if (P) P[i] = ri->GetPressure(i);
  }
}
int ref_remdinfo_exchange(void* h, long step, const double* pot, const double* vol,
                          const double* u, int* accepted) {
  REMDInfo* ri = static_cast<REMDInfo*>(h);
  ri->SetAllIsExchangedGlobal(false);
  const int ec_type = step % 4;
  const int len = ri->GetListLength(ec_type);
  for (int i = 0; i < len; ++i) {
    const Pair pair = ri->GetPair(ec_type, i);
    const int ind1 = ri->GetIndex(pair.a);
    const int ind2 = ri->GetIndex(pair.b);
    const double beta1 = 1. / ri->GetTemperature(ind1);
    const double beta2 = 1. / ri->GetTemperature(ind2);
    const double press1 = ri->GetPressure(ind1);
    const double press2 = ri->GetPressure(ind2);
    double delta = (beta2 - beta1) * (pot[ind1] - pot[ind2]);
    if (((ri->GetEnsemble() >> PSHIFT) & MASK) > 0)
      delta += (beta2 * press2 - beta1 * press1) * (vol[ind1] - vol[ind2]);
    if (exp(-delta) > u[i]) {
      ri->ExchangeAccepted(ec_type, i);
      accepted[i] = 1;
    } else {
      ri->ExchangeRejected(ec_type, i);
      accepted[i] = 0;
    }
  }
  return len;
}

// ---- (volume, potential) histograms of the compiled REMDInfo ----
// Conditions and the condition-slot -> replica index, set from outside (the
// exchange that moves them is pinned separately).
void ref_remdinfo_set_arrays(void* h, const int* index, const double* T, const double* P) {
  REMDInfo* ri = static_cast<REMDInfo*>(h);
  for (int i = 0; i < ri->GetNumReplica(); i++) {
    ri->index[i] = index[i];
    ri->temperature[i] = T[i];
    ri->pressure[i] = P[i];
  }
}
// REMD::IncrementHistogram (src/remd.cxx:803-813) restated around the compiled
// REMDInfo::IncrementHistogram / KeepAverages; ave = 19 Average fields per replica.
void ref_remdinfo_increment_histogram(void* h, const double* pot, const double* vol, const double* ave) {
  REMDInfo* ri = static_cast<REMDInfo*>(h);
  for (int i = 0; i < ri->GetNumReplica(); ++i) {
    const int ind = ri->GetIndex(i);
    const double p = pot[ind] / (double)ri->GetNmol();
    const double v = vol[ind] / (double)ri->GetNmol();
    ri->IncrementHistogram(v, p, i);
    Average a;
    for (int k = 0; k < Average::NUM_ELEM; k++) a.sum[k] = ave[ind * Average::NUM_ELEM + k];
    ri->KeepAverages(v, p, i, a);
  }
}
void ref_remdinfo_output_histogram(void* h) { static_cast<REMDInfo*>(h)->OutputHistogram(); }
void ref_remdinfo_read_histogram(void* h) { static_cast<REMDInfo*>(h)->ReadHistogramFromBackUp(); }

// The reference's .gro writer (src/gro.cxx:118-135) on atoms given as arrays:
// molecule id, molecule name, atom name, atom id, coordinates (nm); velocities 0.
void ref_write_gro(const char* path, int natom, const int* molid, const char* const* molname,
                   const char* const* atomname, const int* atomid, const double* coor, const double* L,
                   const char* comment) {
  std::vector<AtomGro> a(natom);
  for (int i = 0; i < natom; i++) {
    std::snprintf(a[i].MolName, sizeof(a[i].MolName), "%s", molname[i]);
    std::snprintf(a[i].AtomName, sizeof(a[i].AtomName), "%s", atomname[i]);
    a[i].MolID = molid[i];
    a[i].AtomID = atomid[i];
    for (int d = 0; d < 3; d++) {
      a[i].coor[d] = coor[3 * i + d];
      a[i].vel[d] = 0.0;
    }
  }
  dvec3 box;
  for (int d = 0; d < 3; d++) box[d] = L[d];
  write_gro_file(path, natom, a.data(), box, comment);
}

}  // extern "C"
