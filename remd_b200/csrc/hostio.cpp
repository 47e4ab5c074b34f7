// hostio.cpp -- host-side formats and decisions of the REMD engine:
//   * the wall table (ForceCalculator::CalcWallForce, src/force_calculator.cxx:117-200),
//     built on the host exactly as the reference builds it (single-precision
//     sqrtf/powf inside the FP64 loop) so the table agrees bit for bit;
//   * the .chk checkpoint reader/writer (src/io_manager.cxx:528-634);
//   * the Metropolis T/P exchange (src/remd.cxx:467-538, src/remdinfo.cxx:54-125).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "../../include/remd_b200.h"
#include "hostio.h"

namespace remd {

static thread_local std::string g_last_error;
void set_error(const std::string& s) { g_last_error = s; }
const char* last_error() { return g_last_error.c_str(); }

// reduced units, src/unit.h:1-19
const double kNa = 6.0221367e+23;
const double kE0 = 8.8542e-12;
const double kEle = 1.6021761e-19;
const double kKB = 1.3806488e-23;
double unit_mass() { return 15.9994e-3 / kNa; }
double unit_length() { return 1.0e-10; }
double unit_energy() { return 1e3 / kNa; }
double unit_time() { return std::sqrt(unit_mass() * unit_length() * unit_length() / unit_energy()); }
double unit_coulomb() { return std::sqrt(4. * M_PI * kE0 * unit_energy() * unit_length()); }
double elementary_charge() { return kEle; }
double unit_temp() { return unit_energy() / kKB; }
double unit_press() { return unit_energy() / (unit_length() * unit_length() * unit_length()); }

void wall_table(int confined, int nfwall, double wall_A, double sgm_A, double eps_kJ, double rho,
                double* fw) {
  const double wall_length = wall_A * 1e-10 / unit_length();
  const double sgm_wall = sgm_A * 1e-10 / unit_length();
  const double eps_wall = eps_kJ * 1e3 / kNa / unit_energy();
  const double dr = wall_length / (double)nfwall;
  if (confined == 1) {
    const int ninteg = 10000;
    const double dphi = M_PI / (double)ninteg;
    const double sgm06 = powf((float)sgm_wall, 6);
    const double R02 = wall_length * wall_length;
    // the phi integral per table entry is independent: split entries over threads
    unsigned nth = std::thread::hardware_concurrency();
    if (nth < 1) nth = 1;
    if (nth > 32) nth = 32;
    if ((long long)nfwall * ninteg < 4000000LL) nth = 1;
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < nth; t++) {
      pool.emplace_back([=]() {
        for (int i = (int)t; i < nfwall; i += (int)nth) {
          const double r = (double)i * dr;
          const double r02 = r * r;
          double tmp, sum = 0.0;
          for (int j = 0; j < ninteg; j++) {
            const double phi = M_PI - (double)j * dphi;
            const double rho_min = sqrtf((float)(R02 + r02 - 2.0 * wall_length * r * std::cos(phi)));
            const double rho_mini = 1.0 / rho_min;
            const double rho_min05i = rho_mini * rho_mini * rho_mini * rho_mini * rho_mini;
            tmp = 63.0 / 32.0 * sgm06 * rho_min05i * rho_min05i * rho_mini;
            tmp -= 3.0 * rho_min05i;
            sum += tmp;
          }
          fw[2 * i + 1] = M_PI * rho * eps_wall * sgm06 * sum * wall_length * dphi;
        }
      });
    }
    for (auto& th : pool) th.join();
    for (int i = 1; i < nfwall - 1; i++) {
      const double r = (double)i * dr;
      fw[2 * i] = -(fw[2 * (i + 1) + 1] - fw[2 * (i - 1) + 1]) / (2.0 * dr * r);
    }
    fw[0] = fw[2];
    fw[2 * (nfwall - 1)] = (fw[2 * (nfwall - 2)] - fw[2 * (nfwall - 3)]) * 2.0 + fw[2 * (nfwall - 3)];
  } else if (confined == 2) {
    for (int i = 0; i < nfwall; i++) {
      const double rd = 0.5 * wall_length + 0.5 * (double)i * dr;
      const double rdi = 1.0 / rd;
      const double ru = 0.5 * wall_length - 0.5 * (double)i * dr;
      const double rui = 1.0 / ru;
      const double rd03i = rdi * rdi * rdi, rd06i = rd03i * rd03i;
      const double ru03i = rui * rui * rui, ru06i = ru03i * ru03i;
      double f = (9.0 * eps_wall * rd06i * rd03i - 3.0 * sgm_wall * rd03i) * rdi;
      f -= (9.0 * eps_wall * ru06i * ru03i - 3.0 * sgm_wall * ru03i) * rui;
      double u = eps_wall * rd06i * rd03i - sgm_wall * rd03i;
      u += eps_wall * ru06i * ru03i - sgm_wall * ru03i;
      fw[2 * i] = f;
      fw[2 * i + 1] = u;
    }
  }
}

int exchange_host(int nt, int np, int pconstant, long step, int* index, double* T, double* P,
                  const double* pot, const double* vol, const double* u, int* accepted) {
  int pair = 0;
  auto trial = [&](int a, int b) {
    const int i1 = index[a], i2 = index[b];
    const double b1 = 1. / T[i1], b2 = 1. / T[i2];
    double delta = (b2 - b1) * (pot[i1] - pot[i2]);
    if (pconstant > 0) delta += (b2 * P[i2] - b1 * P[i1]) * (vol[i1] - vol[i2]);
    const bool acc = std::exp(-delta) > u[pair];
    if (acc) {
      std::swap(T[index[a]], T[index[b]]);
      std::swap(P[index[a]], P[index[b]]);
      std::swap(index[a], index[b]);
    }
    if (accepted) accepted[pair] = acc ? 1 : 0;
    pair++;
  };
  switch ((int)(step % 4)) {
    case 0:
      for (int j = 0; j < np; ++j)
        for (int i = 0; i < nt / 2; ++i) trial(2 * i + j * nt, 2 * i + 1 + j * nt);
      break;
    case 1:
      for (int j = 0; j < np / 2; ++j)
        for (int i = 0; i < nt; ++i) trial(i + 2 * j * nt, i + (2 * j + 1) * nt);
      break;
    case 2:
      for (int j = 0; j < np; ++j)
        for (int i = 0; i < nt / 2 - (nt + 1) % 2; ++i) trial(2 * i + j * nt + 1, 2 * i + 1 + j * nt + 1);
      break;
    default:
      for (int j = 0; j < np / 2 - (np + 1) % 2; ++j)
        for (int i = 0; i < nt; ++i) trial(i + (2 * j + 1) * nt, i + (2 * j + 2) * nt);
      break;
  }
  return pair;
}

int exchange_pair_count(int nt, int np, long step) {
  switch ((int)(step % 4)) {
    case 0: return np * (nt / 2);
    case 1: return (np / 2) * nt;
    case 2: return np * std::max(0, nt / 2 - (nt + 1) % 2);
    default: return std::max(0, np / 2 - (np + 1) % 2) * nt;
  }
}

int read_chk(const char* path, int nmol, double* r, double* v, double* q, double* p, double* mass,
             double* inertia, double* scal) {
  std::ifstream is(path);
  if (!is) {
    set_error(std::string("cannot open ") + path);
    return REMD_ERR_IO;
  }
  int n = 0, na = 0;
  is >> n >> na;
  if (!is || n != nmol) {
    set_error("chk: molecule count mismatch");
    return REMD_ERR_INVALID;
  }
  std::vector<double> rows((size_t)n * 18);
  for (int i = 0; i < n; i++) {
    for (int k = 0; k < 18; k++) is >> rows[(size_t)i * 18 + k];
    int type, id;
    is >> type >> id;
  }
  double s, Ps, Q, Pv[3], W, L[3];
  is >> s >> Ps >> Q >> Pv[0] >> Pv[1] >> Pv[2] >> W >> L[0] >> L[1] >> L[2];
  if (!is) {
    set_error("chk: truncated file");
    return REMD_ERR_IO;
  }
  for (int i = 0; i < n; i++) {
    const double* w = &rows[(size_t)i * 18];
    for (int d = 0; d < 3; d++) {
      r[3 * i + d] = w[d] / L[d];
      v[3 * i + d] = w[3 + d] * (L[d] * s);
      inertia[3 * i + d] = w[15 + d];
    }
    for (int d = 0; d < 4; d++) {
      q[4 * i + d] = w[6 + d];
      p[4 * i + d] = w[10 + d] * s;
    }
    mass[i] = w[14];
  }
  const double sc[10] = {s, Ps, Q, Pv[0], Pv[1], Pv[2], W, L[0], L[1], L[2]};
  std::memcpy(scal, sc, sizeof(sc));
  return REMD_OK;
}

// The stream formats of the reference: Vector's operator<< writes ' ' then each
// component in std::scientific (src/vector.h:141-147), which stays in effect for
// the scalars after it; Property's operator<< writes its first eleven scalars
// with std::setw(10) (no padding for a finite %e, 12+ characters), each followed
// by ' ', then Vector and scalar fields each followed by ' ' (src/variables.h:51-74).
int write_chk(const char* path, int nmol, int nsite, const double* r, const double* v,
              const double* q, const double* p, double mass, const double* I, double s, double Ps,
              double Q, const double* Pv, double W, const double* L, const double* prop) {
  if (!prop) {
    set_error("chk: the Property line's values are missing");
    return REMD_ERR_INVALID;
  }
  FILE* f = std::fopen(path, "w");
  if (!f) {
    set_error(std::string("cannot write ") + path);
    return REMD_ERR_IO;
  }
  std::fprintf(f, "%d %d\n", nmol, nmol * nsite);
  for (int i = 0; i < nmol; i++) {
    for (int d = 0; d < 3; d++) {
      if (r[3 * i + d] < 0.0 || r[3 * i + d] > 1.0) {
        std::fclose(f);
        set_error("chk: molecule out of box");   // src/io_manager.cxx:614-617
        return REMD_ERR_INVALID;
      }
    }
    for (int d = 0; d < 3; d++) std::fprintf(f, " %e", r[3 * i + d] * L[d]);
    for (int d = 0; d < 3; d++) std::fprintf(f, " %e", v[3 * i + d] / (L[d] * s));
    for (int d = 0; d < 4; d++) std::fprintf(f, " %e", q[4 * i + d]);
    for (int d = 0; d < 4; d++) std::fprintf(f, " %e", p[4 * i + d] / s);
    std::fprintf(f, " %e  %e %e %e 0 %d\n", mass, I[0], I[1], I[2], i * nsite);
  }
  std::fprintf(f, "%e %e %e\n", s, Ps, Q);
  std::fprintf(f, " %e %e %e %e\n", Pv[0], Pv[1], Pv[2], W);
  std::fprintf(f, " %e %e %e\n", L[0], L[1], L[2]);
  // the Property line: time ... ham, tmo, Tave, prs, vir, Pave
  for (int k = 0; k < 11; k++) std::fprintf(f, "%10e ", prop[k]);
  for (int k = 11; k < 14; k++) std::fprintf(f, " %e", prop[k]);
  std::fprintf(f, " %e ", prop[14]);
  for (int k = 15; k < 19; k++) std::fprintf(f, " %e", prop[k]);
  std::fprintf(f, " ");
  for (int k = 19; k < 22; k++) std::fprintf(f, " %e", prop[k]);
  std::fprintf(f, " ");
  for (int k = 22; k < 26; k++) std::fprintf(f, " %e", prop[k]);
  std::fprintf(f, " \n");
  if (std::fclose(f) != 0) {
    set_error(std::string("chk: write failed: ") + path);
    return REMD_ERR_IO;
  }
  return REMD_OK;
}

}  // namespace remd

extern "C" {

const char* remd_last_error(void) { return remd::last_error(); }
const char* remd_version(void) { return "remd_b200 0.1 (sm_100a)"; }

remd_status remd_wall_table(int confined, int nfwall, double wall_length, double sgm_wall,
                            double eps_wall, double rho_wall, double* out) {
  if (!out || nfwall < 3 || (confined != 1 && confined != 2) || wall_length <= 0.0) {
    remd::set_error("remd_wall_table: confined must be 1 or 2, nfwall >= 3, wall_length > 0");
    return REMD_ERR_INVALID;
  }
  remd::wall_table(confined, nfwall, wall_length, sgm_wall, eps_wall, rho_wall, out);
  return REMD_OK;
}

remd_status remd_exchange_host(int ntemp, int npress, int pconstant, long step, int* index,
                               double* temperature, double* pressure, const double* pot,
                               const double* vol, const double* u, int* accepted, int* npairs) {
  if (ntemp < 1 || npress < 1 || !index || !temperature || !pressure || !pot || !vol || !u) {
    remd::set_error("remd_exchange_host: bad arguments");
    return REMD_ERR_INVALID;
  }
  const int n = remd::exchange_host(ntemp, npress, pconstant, step, index, temperature, pressure,
                                    pot, vol, u, accepted);
  if (npairs) *npairs = n;
  return REMD_OK;
}

remd_status remd_read_chk(const char* path, int nmol, double* r, double* v, double* q, double* p,
                          double* mass, double* inertia, double* scal) {
  if (!path || nmol < 1 || !r || !v || !q || !p || !mass || !inertia || !scal) {
    remd::set_error("remd_read_chk: bad arguments");
    return REMD_ERR_INVALID;
  }
  return (remd_status)remd::read_chk(path, nmol, r, v, q, p, mass, inertia, scal);
}

remd_status remd_write_chk_arrays(const char* path, int nmol, int nsite, const double* r,
                                  const double* v, const double* q, const double* p, double mass,
                                  const double* inertia, const double* scal, const double* prop) {
  if (!path || nmol < 1 || nsite < 1 || !r || !v || !q || !p || !inertia || !scal || !prop) {
    remd::set_error("remd_write_chk_arrays: bad arguments");
    return REMD_ERR_INVALID;
  }
  return (remd_status)remd::write_chk(path, nmol, nsite, r, v, q, p, mass, inertia, scal[0], scal[1],
                                      scal[2], scal + 3, scal[6], scal + 7, prop);
}

}  // extern "C"
