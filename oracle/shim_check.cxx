// shim_check.cxx -- drives the engine through the REMDGPU shim
// (remd_b200/shim/remdgpu.h) from the reference's own Molecules objects, next to
// the reference's CPU Molecules::ExecuteSteps on copies of the same replicas.
// TEST INFRASTRUCTURE ONLY (built by oracle/Makefile into oracle/_ref/).
//
// usage: shim_check <inp file> <chk file> <intervals>
// prints one line per replica and interval: "rep <r> <k> gpu <19 averages> cpu <19 averages>"
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <vector>

#include "remdgpu.h"

static void load(Molecules* m, const char* chk) {
  const int n = m->nmol;
  std::vector<double> r(3 * n), v(3 * n), q(4 * n), p(4 * n), mass(n), I(3 * n), sc(10);
  if (remd_read_chk(chk, n, r.data(), v.data(), q.data(), p.data(), mass.data(), I.data(), sc.data()) != REMD_OK) {
    std::fprintf(stderr, "chk: %s\n", remd_last_error());
    std::exit(1);
  }
  for (int i = 0; i < n; i++) {
    for (int x = 0; x < 3; x++) {
      m->mlcl[i].r[x] = r[3 * i + x];
      m->mlcl[i].v[x] = v[3 * i + x];
      m->mlcl[i].i[x] = I[3 * i + x];
    }
    for (int x = 0; x < 4; x++) {
      m->mlcl[i].q[x] = q[4 * i + x];
      m->mlcl[i].p[x] = p[4 * i + x];
    }
    m->mlcl[i].m = mass[i];
    m->mlcl[i].type = 0;
    m->mlcl[i].id = i * (int)m->mlist[0].a.size();
  }
  m->tst->s = sc[0]; m->tst->Ps = sc[1]; m->tst->Q = sc[2];
  for (int x = 0; x < 3; x++) { m->bst->Pv[x] = sc[3 + x]; m->L[x] = sc[7 + x]; }
  m->bst->W = sc[6];
}

int main(int argc, char** argv) {
  if (argc < 4) return 2;
  Parameter prm;
  std::ifstream f(argv[1]);
  prm.read(f);
  const int nrep = prm.nreplica, nint = std::atoi(argv[3]);
  // REMDInfo's destructor deletes its Histogram objects with delete[]
  // (src/remdinfo.cxx:296-300): keep it alive until the process ends.
  REMDInfo& info = *new REMDInfo(prm);
  std::vector<Molecules*> gpu(nrep), cpu(nrep);
  for (int k = 0; k < nrep; k++) {
    for (Molecules** mm : {&gpu[k], &cpu[k]}) {
      *mm = new Molecules(prm);
      Molecules* m = *mm;
      load(m, argv[2]);
      m->SetTemperature(info.GetTemperature(k));
      m->SetPressure(info.GetPressure(k));
      if (prm.init_scaling == 1) { m->VelocityScaling(); m->AngVelocityScaling(); }
      if (prm.tstat_mass > 0.0) { m->tst->Q = prm.tstat_mass; m->tst->flush(); }
      m->InitializeProperty();
    }
  }
  REMDGPU eng(gpu.data(), nrep);
  for (int s = 0; s < nint; s++) {
    eng.ExecuteSteps(info.temperature, info.pressure);
    for (int k = 0; k < nrep; k++) {
      cpu[k]->ExecuteSteps();
      Average a = eng.GetAverages(k);
      Average b = cpu[k]->GetAverage();
      std::printf("rep %d %d gpu", k, s);
      for (int i = 0; i < 18; i++) std::printf(" %.17g", a.sum[i]);
      std::printf(" cpu");
      for (int i = 0; i < 18; i++) std::printf(" %.17g", b.sum[i]);
      std::printf("\n");
    }
  }
  eng.ConvertVariablesToHost(gpu.data());
  std::printf("state L %.17g %.17g %.17g s %.17g\n", gpu[0]->L[0], gpu[0]->L[1], gpu[0]->L[2], gpu[0]->tst->s);
  std::fflush(stdout);
  std::_Exit(0);   // the reference's destructors free memory they never allocated
}
