// hostio.h -- host-side helpers shared by the engine translation units.
#pragma once
#include <string>

namespace remd {

void set_error(const std::string& s);
const char* last_error();

double unit_mass();
double unit_length();
double unit_energy();
double unit_time();
double unit_coulomb();
double elementary_charge();   // C, src/unit.h
double unit_temp();
double unit_press();

void wall_table(int confined, int nfwall, double wall_A, double sgm_A, double eps_kJ, double rho,
                double* fw);
int exchange_host(int nt, int np, int pconstant, long step, int* index, double* T, double* P,
                  const double* pot, const double* vol, const double* u, int* accepted);
int exchange_pair_count(int nt, int np, long step);
int read_chk(const char* path, int nmol, double* r, double* v, double* q, double* p, double* mass,
             double* inertia, double* scal);
// IOManager::WriteCheckPoint (src/io_manager.cxx:593-634).  prop: the 26
// numbers of its last line, in Property's operator<< order (src/variables.h:
// 51-74): time pot tra rot kin tsm tsp tst bst tot ham, tmo[3], Tave (already
// divided by nave), prs[4], vir[3], Pave[4] (divided by nave).
constexpr int kChkPropCount = 26;
int write_chk(const char* path, int nmol, int nsite, const double* r, const double* v,
              const double* q, const double* p, double mass, const double* I, double s, double Ps,
              double Q, const double* Pv, double W, const double* L, const double* prop);

}  // namespace remd
