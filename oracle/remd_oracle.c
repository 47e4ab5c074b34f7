/*
 * remd_oracle.c -- FP64 CPU restatement of the subarutaro/remd hot path.
 * TEST INFRASTRUCTURE ONLY (the parity checker); the engine never links it.
 *
 * Every function follows the reference file:line named in its comment, with
 * the same floating-point operation order, so that a build with the same
 * compiler flags as oracle/_ref agrees with the reference to rounding.
 * Deliberate departures from the reference CPU code:
 *   - the cylinder table lookup clamps its base index to nfwall-2 instead of
 *     reading one entry past the table (src/force_calculator.cxx:1549-1551);
 *   - confined=2 (slit) follows the reference GPU kernel: wall force
 *     src/remdgpu.cu:1708-1720, D5 src/remdgpu.cu:2537-2545, D4 2096-2115,
 *     barostat energy src/remdgpu.cu:2803-2809.  Pressure mode 3 always uses
 *     that GPU form.
 */
#include "remd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---- units: src/unit.h:1-19 ---- */
static const double kNa = 6.0221367e+23;
static const double kE0 = 8.8542e-12;
static const double kEle = 1.6021761e-19;
static const double kKB = 1.3806488e-23;

static double u_mass(void) { return 15.9994e-3 / kNa; }
static double u_length(void) { return 1.0e-10; }
static double u_energy(void) { return 1e3 / kNa; }
double orc_unit_mass(void) { return u_mass(); }
double orc_unit_time(void) { return sqrt(u_mass() * u_length() * u_length() / u_energy()); }
double orc_unit_coulomb(void) { return sqrt(4. * M_PI * kE0 * u_energy() * u_length()); }
double orc_unit_temp(void) { return u_energy() / kKB; }
double orc_unit_press(void) { return u_energy() / (u_length() * u_length() * u_length()); }

#define TMODE(s) ((s)->tconstant)
#define PMODE(s) ((s)->pconstant)
#define CMODE(s) ((s)->confined)

/* ---- molecule type: src/molecules.cxx:95-109, src/variables.h:316-334,
 *      src/force_calculator.cxx:219-233 ---- */
void orc_moltype_from_input(orc_moltype *mt, int nsite, const double *r,
                            const double *mass, const double *sigma,
                            const double *eps, const double *charge) {
  memset(mt, 0, sizeof(*mt));
  mt->nsite = nsite;
  double s[ORC_NSITE_MAX], e[ORC_NSITE_MAX];
  for (int k = 0; k < nsite; k++) {
    for (int d = 0; d < 3; d++) mt->body[k][d] = r[3 * k + d] * (1e-10 / u_length());
    mt->mass[k] = mass[k] * (1e-03 / kNa / u_mass());
    s[k] = sigma[k] * (1e-10 / u_length());
    e[k] = eps[k] * (1e+03 / kNa / u_energy());
    mt->q[k] = charge[k] * (kEle / orc_unit_coulomb());
  }
  for (int i = 0; i < nsite; i++)
    for (int j = 0; j < nsite; j++) {
      double sg = 0.5 * (s[i] + s[j]);
      mt->sgm2[i][j] = sg * sg;
      mt->eps[i][j] = sqrt(e[i] * e[j]);
    }
  double xx = 0, yy = 0, zz = 0;
  for (int k = 0; k < nsite; k++) {
    double m = mt->mass[k], x = mt->body[k][0], y = mt->body[k][1], z = mt->body[k][2];
    xx += m * (y * y + z * z);
    yy += m * (z * z + x * x);
    zz += m * (x * x + y * y);
  }
  mt->inertia[0] = xx;
  mt->inertia[1] = yy;
  mt->inertia[2] = zz;
}

/* Molecules ctor (src/molecules.h:89-93) and ForceCalculator ctor (src/force_calculator.cxx:15-50). */
void orc_system_init(orc_system *sys, int nmol, int tconstant, int pconstant,
                     int confined, double dt_fs, double rcut, double rswitch,
                     int nfwall, double wall_length_A) {
  sys->nmol = nmol;
  sys->tconstant = tconstant;
  sys->pconstant = pconstant;
  sys->confined = confined;
  sys->dt = dt_fs * 1e-15 / orc_unit_time();
  sys->dthalf = dt_fs * 1e-15 / orc_unit_time() * 0.5;
  sys->rcut = rcut;
  sys->rswitch = rswitch;
  sys->nfwall = nfwall;
  sys->wall_length_param = wall_length_A;
  sys->wall_length = wall_length_A * 1e-10 / u_length();
}

/* ---- rotations: src/rotation.h:146-187 ---- */
static void body_to_space(const double *a, const double *v, double *out) {
  const double a0sq = a[0] * a[0], a1sq = a[1] * a[1], a2sq = a[2] * a[2], a3sq = a[3] * a[3];
  const double a01 = a[0] * a[1], a02 = a[0] * a[2], a03 = a[0] * a[3];
  const double a12 = a[1] * a[2], a13 = a[1] * a[3], a23 = a[2] * a[3];
  double t0 = (a0sq + a1sq - a2sq - a3sq) * v[0];
  t0 += 2. * (a12 - a03) * v[1];
  t0 += 2. * (a13 + a02) * v[2];
  double t1 = 2. * (a12 + a03) * v[0];
  t1 += (a0sq - a1sq + a2sq - a3sq) * v[1];
  t1 += 2. * (a23 - a01) * v[2];
  double t2 = 2. * (a13 - a02) * v[0];
  t2 += 2. * (a23 + a01) * v[1];
  t2 += (a0sq - a1sq - a2sq + a3sq) * v[2];
  out[0] = t0; out[1] = t1; out[2] = t2;
}

static void space_to_body(const double *a, const double *v, double *out) {
  const double a0sq = a[0] * a[0], a1sq = a[1] * a[1], a2sq = a[2] * a[2], a3sq = a[3] * a[3];
  const double a01 = a[0] * a[1], a02 = a[0] * a[2], a03 = a[0] * a[3];
  const double a12 = a[1] * a[2], a13 = a[1] * a[3], a23 = a[2] * a[3];
  double t0 = (a0sq + a1sq - a2sq - a3sq) * v[0];
  t0 += 2. * (a12 + a03) * v[1];
  t0 += 2. * (a13 - a02) * v[2];
  double t1 = 2. * (a12 - a03) * v[0];
  t1 += (a0sq - a1sq + a2sq - a3sq) * v[1];
  t1 += 2. * (a23 + a01) * v[2];
  double t2 = 2. * (a13 + a02) * v[0];
  t2 += 2. * (a23 - a01) * v[1];
  t2 += (a0sq - a1sq - a2sq + a3sq) * v[2];
  out[0] = t0; out[1] = t1; out[2] = t2;
}

/* P1/P2/P3 and S(q): src/integrator.h:103-160 */
static void P1(const double *q, double *o) { o[0] = -q[1]; o[1] = q[0]; o[2] = q[3]; o[3] = -q[2]; }
static void P2(const double *q, double *o) { o[0] = -q[2]; o[1] = -q[3]; o[2] = q[0]; o[3] = q[1]; }
static void P3(const double *q, double *o) { o[0] = -q[3]; o[1] = q[2]; o[2] = -q[1]; o[3] = q[0]; }
static double dot4(const double *a, const double *b) {
  double t = 0.0;
  for (int k = 0; k < 4; k++) t += a[k] * b[k];
  return t;
}

/* ---- wall table: ForceCalculator::CalcWallForce, src/force_calculator.cxx:117-200 ---- */
void orc_wall_table(int confined, int nfwall, double wall_A, double sgm_A, double eps_kJ,
                    double rho, double *fwall) {
  const double wall_length = wall_A * 1e-10 / u_length();
  const double sgm_wall = sgm_A * 1e-10 / u_length();
  const double eps_wall = eps_kJ * 1e3 / kNa / u_energy();
  const double rho_wall = rho;
  const double dr = wall_length / (double)nfwall;
  if (confined == 1) {
    const int ninteg = 10000;
    const double dphi = M_PI / (double)ninteg;
    const double sgm06 = powf((float)sgm_wall, 6);
    const double R02 = wall_length * wall_length;
    for (int i = 0; i < nfwall; i++) {
      const double r = (double)i * dr;
      const double r02 = r * r;
      double tmp, sum = 0.0;
      for (int j = 0; j < ninteg; j++) {
        const double phi = M_PI - (double)j * dphi;
        const double rho_min = sqrtf((float)(R02 + r02 - 2.0 * wall_length * r * cos(phi)));
        const double rho_mini = 1.0 / rho_min;
        const double rho_min05i = rho_mini * rho_mini * rho_mini * rho_mini * rho_mini;
        tmp = 63.0 / 32.0 * sgm06 * rho_min05i * rho_min05i * rho_mini;
        tmp -= 3.0 * rho_min05i;
        sum += tmp;
      }
      fwall[2 * i + 1] = M_PI * rho_wall * eps_wall * sgm06 * sum * wall_length * dphi;
    }
    for (int i = 1; i < nfwall - 1; i++) {
      const double r = (double)i * dr;
      fwall[2 * i + 0] = -(fwall[2 * (i + 1) + 1] - fwall[2 * (i - 1) + 1]) / (2.0 * dr * r);
    }
    fwall[0] = fwall[2];
    fwall[2 * (nfwall - 1)] =
        (fwall[2 * (nfwall - 2)] - fwall[2 * (nfwall - 3)]) * 2.0 + fwall[2 * (nfwall - 3)];
  }
  if (confined == 2) {
    for (int i = 0; i < nfwall; i++) {
      const double rd = 0.5 * wall_length + 0.5 * (double)i * dr;
      const double rdi = 1.0 / rd;
      const double ru = 0.5 * wall_length - 0.5 * (double)i * dr;
      const double rui = 1.0 / ru;
      const double rd03i = rdi * rdi * rdi;
      const double rd06i = rd03i * rd03i;
      const double ru03i = rui * rui * rui;
      const double ru06i = ru03i * ru03i;
      double f = (9.0 * eps_wall * rd06i * rd03i - 3.0 * sgm_wall * rd03i) * rdi;
      f -= (9.0 * eps_wall * ru06i * ru03i - 3.0 * sgm_wall * ru03i) * rui;
      double u = eps_wall * rd06i * rd03i - sgm_wall * rd03i;
      u += eps_wall * ru06i * ru03i - sgm_wall * ru03i;
      fwall[2 * i + 0] = f;
      fwall[2 * i + 1] = u;
    }
  }
}

/* ---- volume: Molecules::GetVolume / GetBottomArea, src/molecules.h:357-376 ---- */
static double bottom_area(const orc_system *sys) {
  const double sigma_c = 3.4;
  const double wl = (sys->wall_length_param - 0.5 * sigma_c) * 1e-10 / u_length();
  return M_PI * wl * wl;
}
double orc_volume(const orc_system *sys, const orc_replica *rep) {
  if (sys->confined == 1) return bottom_area(sys) * rep->L[2];
  if (sys->confined == 2) {
    const double wl = sys->wall_length_param * 1e-10 / u_length();
    return rep->L[0] * rep->L[1] * wl;
  }
  return rep->L[0] * rep->L[1] * rep->L[2];
}

/* ---- force: Molecules::CalcForcePot, src/molecules.cxx:531-629 (generic build) ---- */
static void convert_to_atoms(const orc_system *sys, orc_replica *rep) {
  /* src/molecules.cxx:362-389 */
  const int ns = sys->mt.nsite;
  const double *L = rep->L;
  for (int i = 0; i < sys->nmol; i++) {
    for (int d = 0; d < ns; d++) {
      double b2s[3];
      body_to_space(&rep->q[4 * i], sys->mt.body[d], b2s);
      double *a = &rep->ar[3 * (ns * i + d)];
      for (int k = 0; k < 3; k++) a[k] = rep->r[3 * i + k] * L[k] + b2s[k];
      for (int k = 0; k < 3; k++)
        if (a[k] >= L[k]) a[k] -= L[k];
      for (int k = 0; k < 3; k++)
        if (a[k] < 0) a[k] += L[k];
      double *af = &rep->af[3 * (ns * i + d)];
      af[0] = af[1] = af[2] = 0.0;
    }
  }
}

static void switching(const orc_system *sys, orc_replica *rep) {
  /* ForceCalculator::Switching, src/force_calculator.cxx:691-779 */
  const double rc = sys->rcut;
  const double rl = sys->rswitch;
  const double rlc = rl - rc;
  const double coef = 1.0 / (rlc * rlc * rlc * rlc * rlc);
  const double rcutSq = sys->rcut * sys->rcut;
  const int ns = sys->mt.nsite;
  const double *L = rep->L;
  double vir[3] = {0, 0, 0};
  double lj = 0.0, clmb = 0.0;
  long long npairs = 0;
  for (int i = 0; i < sys->nmol; i++) {
    double *fi = &rep->f[3 * i];
    fi[0] = fi[1] = fi[2] = 0.0;
    for (int j = 0; j < sys->nmol; j++) {
      if (i == j) continue;
      double gr[3];
      for (int d = 0; d < 3; d++) gr[d] = (rep->r[3 * i + d] - rep->r[3 * j + d]) * L[d];
      for (int d = 0; d < 3; d++) {
        if (gr[d] >= 0.5 * L[d]) gr[d] -= L[d];
        if (gr[d] < -0.5 * L[d]) gr[d] += L[d];
      }
      double r02 = gr[0] * gr[0] + gr[1] * gr[1] + gr[2] * gr[2];
      if (r02 > rcutSq) continue;
      if (i < j) npairs++;
      const double r01 = sqrt(r02);
      double sw, dsw;
      if (r01 > rl) {
        const double r01c = r01 - rc;
        const double r01l = r01 - rl;
        sw = coef * r01c * r01c * r01c * (10.0 * r01l * r01l - 5.0 * r01l * r01c + r01c * r01c);
        dsw = coef * 30.0 * r01c * r01c * r01l * r01l;
      } else {
        sw = 1.0;
        dsw = 0.0;
      }
      double dswr[3];
      for (int d = 0; d < 3; d++) dswr[d] = gr[d] * (dsw / r01);
      for (int ii = 0; ii < ns; ii++) {
        const double *ari = &rep->ar[3 * (ns * i + ii)];
        double *afi = &rep->af[3 * (ns * i + ii)];
        double e = 0.0;
        double f[3] = {0.0, 0.0, 0.0};
        for (int jj = 0; jj < ns; jj++) {
          const double *arj = &rep->ar[3 * (ns * j + jj)];
          const double qq = sys->mt.q[ii] * sys->mt.q[jj];
          double r[3];
          for (int d = 0; d < 3; d++) r[d] = ari[d] - arj[d];
          for (int d = 0; d < 3; d++) {
            if (r[d] >= 0.5 * L[d]) r[d] -= L[d];
            if (r[d] < -0.5 * L[d]) r[d] += L[d];
          }
          const double rr = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
          const double r02i = 1.0 / rr;
          const double r01i = sqrt(r02i);
          double rs06i = sys->mt.sgm2[ii][jj] * r02i;
          rs06i = rs06i * rs06i * rs06i;
          const double ep = sys->mt.eps[ii][jj];
          const double elj = 4.0 * ep * rs06i * (rs06i - 1.0);
          const double ecl = qq * r01i;
          lj += sw * elj;
          clmb += sw * ecl;
          const double etmp = elj + ecl;
          const double ftmp = (48.0 * ep * rs06i * (rs06i - 0.5) * r02i + qq * r01i * r02i) * sw;
          e += etmp;
          for (int d = 0; d < 3; d++) f[d] += r[d] * ftmp;
          for (int d = 0; d < 3; d++) afi[d] += r[d] * ftmp;
        }
        for (int d = 0; d < 3; d++) f[d] -= dswr[d] * e;
        for (int d = 0; d < 3; d++) fi[d] += f[d];
        for (int d = 0; d < 3; d++) vir[d] += f[d] * gr[d];
      }
    }
  }
  for (int d = 0; d < 3; d++) rep->vir[d] = vir[d] * 0.5;
  rep->lj = lj * 0.5;
  rep->clmb = clmb * 0.5;
  rep->npairs = npairs;
}

static void confined(const orc_system *sys, orc_replica *rep) {
  /* ForceCalculator::Confined, generic branch, src/force_calculator.cxx:1527-1566;
   * slit per src/remdgpu.cu:1708-1720 */
  const int ns = sys->mt.nsite;
  const double dr = sys->wall_length / (double)sys->nfwall;
  const double *L = rep->L;
  const double *fw = sys->fwall;
  double wall = 0.0;
  for (int i = 0; i < sys->nmol; i++) {
    const double *a = &rep->ar[3 * (ns * i)];   /* site 0 = oxygen (atom type 0) */
    double *af = &rep->af[3 * (ns * i)];
    if (sys->confined == 1) {
      double r_i[3];
      for (int d = 0; d < 3; d++) r_i[d] = a[d] - L[d] * 0.5;
      const double r01 = sqrt(r_i[0] * r_i[0] + r_i[1] * r_i[1]);
      int index = (int)(r01 / dr);
      if (index > sys->nfwall - 2) index = sys->nfwall - 2;
      const double f = (fw[2 * (index + 1)] - fw[2 * index]) / dr * (r01 - dr * index) + fw[2 * index];
      const double e = (fw[2 * (index + 1) + 1] - fw[2 * index + 1]) / dr * (r01 - dr * index) + fw[2 * index + 1];
      af[0] += f * r_i[0];
      af[1] += f * r_i[1];
      rep->f[3 * i + 0] += f * r_i[0];
      rep->f[3 * i + 1] += f * r_i[1];
      wall += e;
    } else if (sys->confined == 2) {
      const double z = a[2] - 0.5 * L[2];
      const double za = fabs(z);
      const double dir = (za != 0.0) ? z / za : 1.0;
      const double hdr = 0.5 * dr;
      int index = (int)(za / hdr);
      if (index > sys->nfwall - 2) index = sys->nfwall - 2;
      const double f = (fw[2 * (index + 1)] - fw[2 * index]) / hdr * (za - hdr * index) + fw[2 * index];
      const double e = (fw[2 * (index + 1) + 1] - fw[2 * index + 1]) / hdr * (za - hdr * index) + fw[2 * index + 1];
      af[2] += f * dir;
      rep->f[3 * i + 2] += f * dir;
      wall += e;
    }
  }
  rep->wall = wall;
}

static void convert_from_atoms(const orc_system *sys, orc_replica *rep) {
  /* src/molecules.cxx:447-475 (SWITCHING: molecule force comes from the pair loop) */
  const int ns = sys->mt.nsite;
  for (int i = 0; i < sys->nmol; i++) {
    double n[4] = {0, 0, 0, 0};
    for (int d = 0; d < ns; d++) {
      const double *af = &rep->af[3 * (ns * i + d)];
      const double *b = sys->mt.body[d];
      double fb[3];
      space_to_body(&rep->q[4 * i], af, fb);
      n[0] += b[0] * fb[0] + b[1] * fb[1] + b[2] * fb[2];
      n[1] += b[1] * fb[2] - b[2] * fb[1];
      n[2] += b[2] * fb[0] - b[0] * fb[2];
      n[3] += b[0] * fb[1] - b[1] * fb[0];
    }
    for (int k = 0; k < 4; k++) rep->n[4 * i + k] = n[k];
  }
  rep->pot = rep->lj + rep->clmb + rep->wall;
}

void orc_force(const orc_system *sys, orc_replica *rep) {
  convert_to_atoms(sys, rep);
  switching(sys, rep);
  rep->wall = 0.0;
  if (sys->confined > 0) confined(sys, rep);
  convert_from_atoms(sys, rep);
}

/* ---- integrator: src/integrator.cxx (AoS variant, one thread, nlane=1) ---- */
static void D6(const orc_system *sys, orc_replica *rep) {
  /* src/integrator.cxx:634-644 */
  if (TMODE(sys) == 1) {
    const double tmp = 1.0 + (rep->Ps / (2.0 * rep->Q) * sys->dthalf);
    rep->s *= tmp * tmp;
    rep->Ps /= tmp;
  }
}

static void D5(const orc_system *sys, orc_replica *rep) {
  /* src/integrator.cxx:564-601; pressure mode 3 per src/remdgpu.cu:2537-2545 */
  const double dthalf = sys->dthalf;
  double coef_v[3];
  for (int d = 0; d < 3; d++) coef_v[d] = rep->L[d] * rep->s * dthalf;
  const double coef_p = 2.0 * rep->s * dthalf;
  for (int i = 0; i < sys->nmol; i++) {
    double *v = &rep->v[3 * i];
    for (int d = 0; d < 3; d++) v[d] += rep->f[3 * i + d] * coef_v[d] / rep->m[i];
    const double *q = &rep->q[4 * i];
    const double *n = &rep->n[4 * i];
    double S[4][4];
    S[0][0] = q[0]; S[0][1] = -q[1]; S[0][2] = -q[2]; S[0][3] = -q[3];
    S[1][0] = q[1]; S[1][1] = q[0];  S[1][2] = -q[3]; S[1][3] = q[2];
    S[2][0] = q[2]; S[2][1] = q[3];  S[2][2] = q[0];  S[2][3] = -q[1];
    S[3][0] = q[3]; S[3][1] = -q[2]; S[3][2] = q[1];  S[3][3] = q[0];
    double *p = &rep->p[4 * i];
    double Sn[4];
    for (int k = 0; k < 4; k++) Sn[k] = dot4(S[k], n);
    for (int k = 0; k < 4; k++) p[k] += Sn[k] * coef_p;
  }
  if (TMODE(sys) == 1) {
    rep->Ps -= rep->pot * dthalf;
    if (PMODE(sys) > 0) rep->Ps -= (rep->P * orc_volume(sys, rep)) * dthalf;
  }
  if (PMODE(sys) == 1) {
    rep->Pv[0] += ((rep->vir[0] + rep->vir[1] + rep->vir[2]) / (3.0 * rep->L[0] * rep->L[1] * rep->L[2]) - rep->P) * rep->s * dthalf;
  }
  if (PMODE(sys) == 2) {
    rep->Pv[2] += rep->s * (rep->vir[2] / rep->L[2] - rep->P * bottom_area(sys)) * dthalf;
  }
  if (PMODE(sys) == 3) {
    const double zlen = (CMODE(sys) == 2) ? sys->wall_length_param : rep->L[2];
    rep->Pv[0] += rep->s * (rep->vir[0] / rep->L[0] - rep->P * rep->L[1] * zlen) * dthalf;
    rep->Pv[1] += rep->s * (rep->vir[1] / rep->L[1] - rep->P * rep->L[0] * zlen) * dthalf;
  }
}

static void D4(const orc_system *sys, orc_replica *rep) {
  /* src/integrator.cxx:604-632; pressure mode 3 per src/remdgpu.cu:2096-2115 */
  const double dthalf = sys->dthalf;
  if (PMODE(sys) == 1) {
    if (TMODE(sys) == 1) rep->Ps -= rep->Pv[0] * rep->Pv[0] / rep->W * dthalf;
    const double V = orc_volume(sys, rep);
    const double Lnew = powf((float)(V + rep->Pv[0] * rep->s / rep->W * dthalf), (float)(1. / 3.));
    rep->L[0] = rep->L[1] = rep->L[2] = Lnew;
  }
  if (PMODE(sys) == 2) {
    if (TMODE(sys) == 1) rep->Ps -= 0.5 * rep->Pv[2] * rep->Pv[2] / rep->W * dthalf;
    rep->L[2] += rep->s * rep->Pv[2] / rep->W * dthalf;
  }
  if (PMODE(sys) == 3) {
    const double bw = 0.5 / rep->W;
    if (TMODE(sys) == 1) rep->Ps -= (rep->Pv[0] * rep->Pv[0] + rep->Pv[1] * rep->Pv[1]) * bw * dthalf;
    rep->L[0] += rep->s * rep->Pv[0] * bw * sys->dt;
    rep->L[1] += rep->s * rep->Pv[1] * bw * sys->dt;
  }
}

/* one free-rotor sub-step about body axis k (1 = x, 2 = y, 3 = z): D1/D2/D3 */
static double rotate(double *q, double *p, int axis, double Ik, double coef_xi, double h) {
  double Pq[4], Pp[4];
  if (axis == 1) { P1(q, Pq); P1(p, Pp); }
  else if (axis == 2) { P2(q, Pq); P2(p, Pp); }
  else { P3(q, Pq); P3(p, Pp); }
  const double xi = dot4(p, Pq) * coef_xi / Ik;
  const double xidt = xi * h;
  const double c = cos(xidt), s = sin(xidt);
  for (int k = 0; k < 4; k++) q[k] = q[k] * c + Pq[k] * s;
  for (int k = 0; k < 4; k++) p[k] = p[k] * c + Pp[k] * s;
  return xi;
}

void orc_step(const orc_system *sys, orc_replica *rep) {
  /* Molecules::ExecuteStep<MODE>, src/integrator.cxx:646-706 */
  const int T1 = (TMODE(sys) == 1);
  const int needPv = (PMODE(sys) > 0 || T1);
  D6(sys, rep);
  D5(sys, rep);
  D4(sys, rep);
  double sum_Pv[3] = {0, 0, 0};
  double sum_Ps = 0.0;
  const double coef_xi = 0.25 / rep->s;
  /* D3 (src/integrator.cxx:540-563) */
  for (int i = 0; i < sys->nmol; i++) {
    const double xi = rotate(&rep->q[4 * i], &rep->p[4 * i], 3, rep->I[3 * i + 2], coef_xi, sys->dthalf);
    if (T1) sum_Ps += 0.5 * xi * xi * rep->I[3 * i + 2];
  }
  /* D2 (src/integrator.cxx:514-538) */
  for (int i = 0; i < sys->nmol; i++) {
    const double xi = rotate(&rep->q[4 * i], &rep->p[4 * i], 2, rep->I[3 * i + 1], coef_xi, sys->dthalf);
    if (T1) sum_Ps += 0.5 * xi * xi * rep->I[3 * i + 1];
  }
  /* D1 (src/integrator.cxx:467-512) */
  {
    const double si = 1.0 / rep->s;
    double coef_r[3];
    for (int d = 0; d < 3; d++) {
      const double Li = 1.0 / rep->L[d];
      coef_r[d] = Li * Li * si * sys->dt;
    }
    const double cxi = 0.25 * si;
    for (int i = 0; i < sys->nmol; i++) {
      double *r = &rep->r[3 * i];
      const double *v = &rep->v[3 * i];
      for (int d = 0; d < 3; d++) r[d] += v[d] * coef_r[d];
      for (int d = 0; d < 3; d++) {
        if (r[d] < 0.0) r[d] += 1.0;
        if (r[d] >= 1.0) r[d] -= 1.0;
      }
      const double xi = rotate(&rep->q[4 * i], &rep->p[4 * i], 1, rep->I[3 * i + 0], cxi, sys->dt);
      if (needPv)
        for (int d = 0; d < 3; d++) sum_Pv[d] += 2.0 * rep->m[i] * v[d] * v[d];
      if (T1) sum_Ps += xi * xi * rep->I[3 * i + 0];
    }
  }
  for (int i = 0; i < sys->nmol; i++) {
    const double xi = rotate(&rep->q[4 * i], &rep->p[4 * i], 2, rep->I[3 * i + 1], coef_xi, sys->dthalf);
    if (T1) sum_Ps += 0.5 * xi * xi * rep->I[3 * i + 1];
  }
  for (int i = 0; i < sys->nmol; i++) {
    const double xi = rotate(&rep->q[4 * i], &rep->p[4 * i], 3, rep->I[3 * i + 2], coef_xi, sys->dthalf);
    if (T1) sum_Ps += 0.5 * xi * xi * rep->I[3 * i + 2];
  }
  /* D3D2D1D2D3_PsPv (src/integrator.cxx:132-172) */
  if (needPv)
    for (int d = 0; d < 3; d++) sum_Pv[d] /= rep->L[d] * rep->L[d] * rep->s * rep->s;
  const double sPv = sum_Pv[0] + sum_Pv[1] + sum_Pv[2];
  if (PMODE(sys) == 1) rep->Pv[0] += rep->s * sPv / (orc_volume(sys, rep) * 3.0) * sys->dthalf;
  if (PMODE(sys) == 2) rep->Pv[2] += rep->s * sum_Pv[2] / rep->L[2] * sys->dthalf;
  if (PMODE(sys) == 3) {
    rep->Pv[0] += rep->s * sum_Pv[0] / rep->L[0] * sys->dthalf;
    rep->Pv[1] += rep->s * sum_Pv[1] / rep->L[1] * sys->dthalf;
  }
  if (T1) rep->Ps += (0.25 * sPv + 2.0 * sum_Ps - (1.0 + log(rep->s)) * rep->gkT + rep->H0) * sys->dt;
  D4(sys, rep);
  orc_force(sys, rep);
  D5(sys, rep);
  D6(sys, rep);
}

/* ---- properties: src/molecules.cxx:631-734 ---- */
static void translational_energy(const orc_system *sys, const orc_replica *rep, double *kin) {
  double coef[3];
  for (int d = 0; d < 3; d++) coef[d] = 1.0 / (rep->L[d] * rep->s);
  kin[0] = kin[1] = kin[2] = 0.0;
  for (int i = 0; i < sys->nmol; i++)
    for (int d = 0; d < 3; d++) kin[d] += (rep->v[3 * i + d] * rep->v[3 * i + d]) * rep->m[i];
  for (int d = 0; d < 3; d++) kin[d] *= coef[d] * coef[d] * 0.5;
}

static double rotational_energy(const orc_system *sys, const orc_replica *rep) {
  const double coef = 0.25 / rep->s;
  double rot[3] = {0, 0, 0};
  for (int i = 0; i < sys->nmol; i++) {
    const double *q = &rep->q[4 * i], *p = &rep->p[4 * i];
    double Pq[4], xi[3];
    P1(q, Pq); xi[0] = dot4(p, Pq);
    P2(q, Pq); xi[1] = dot4(p, Pq);
    P3(q, Pq); xi[2] = dot4(p, Pq);
    for (int k = 0; k < 3; k++) xi[k] *= (1.0 / rep->I[3 * i + k]) * coef;
    for (int k = 0; k < 3; k++) rot[k] += rep->I[3 * i + k] * xi[k] * xi[k] * 2.0;
  }
  return rot[0] + rot[1] + rot[2];
}

static double barostat_energy(const orc_system *sys, const orc_replica *rep) {
  /* Molecules::BarostatEnergy, src/molecules.cxx:663-678; slit per src/remdgpu.cu:2803-2809 */
  if (PMODE(sys) > 0) {
    if (CMODE(sys) == 0)
      return 0.5 * (rep->Pv[0] * rep->Pv[0] + rep->Pv[1] * rep->Pv[1] + rep->Pv[2] * rep->Pv[2]) / rep->W +
             rep->P * rep->L[0] * rep->L[1] * rep->L[2];
    if (CMODE(sys) == 1) return 0.5 * rep->Pv[2] * rep->Pv[2] / rep->W + rep->P * orc_volume(sys, rep);
    return (rep->Pv[0] * rep->Pv[0] + rep->Pv[1] * rep->Pv[1]) * (0.5 / rep->W) + rep->P * orc_volume(sys, rep);
  }
  return 0.0;
}

void orc_calc_properties(const orc_system *sys, orc_replica *rep) {
  double tmp[3];
  translational_energy(sys, rep, tmp);
  for (int d = 0; d < 3; d++) rep->tra3[d] = tmp[d];
  rep->tra = tmp[0] + tmp[1] + tmp[2];
  rep->rot = rotational_energy(sys, rep);
  rep->kin = rep->tra + rep->rot;
  rep->Tk = rep->kin * orc_unit_temp() / (3. * sys->nmol);
  rep->tsm = 0.5 * rep->Ps * rep->Ps / rep->Q;
  rep->tsp = rep->gkT * log(rep->s);
  rep->tst = rep->tsm + rep->tsp;
  rep->bst = barostat_energy(sys, rep);
  rep->tot = rep->pot + rep->kin;
  if (TMODE(sys) == 1) rep->tot += rep->tst;
  if (PMODE(sys) > 0) rep->tot += rep->bst;
  rep->ham = rep->tot - rep->H0;
  const double volume = orc_volume(sys, rep);
  for (int d = 0; d < 3; d++) rep->prs[d] = (tmp[d] * 2.0 + rep->vir[d]) / volume;
  rep->prs[3] = ((tmp[0] * 2.0 + rep->vir[0]) + (tmp[1] * 2.0 + rep->vir[1]) + (tmp[2] * 2.0 + rep->vir[2])) / (3. * volume);
}

void orc_get_average(const orc_system *sys, const orc_replica *rep, double out[ORC_NUM_AVG]) {
  out[0] = rep->lj;
  out[1] = rep->clmb;
  out[2] = rep->wall;
  out[3] = orc_volume(sys, rep);
  out[4] = rep->tra;
  out[5] = rep->rot;
  out[6] = rep->kin / (3.0 * sys->nmol);
  out[7] = rep->prs[3];
  out[8] = rep->prs[0];
  out[9] = rep->prs[1];
  out[10] = rep->prs[2];
  out[11] = rep->tot;
  out[12] = rep->ham;
  out[13] = rep->s;
  out[14] = rep->Ps;
  out[15] = rep->Pv[0];
  out[16] = rep->Pv[1];
  out[17] = rep->Pv[2];
  out[18] = 0.0;
}

void orc_execute_steps(const orc_system *sys, orc_replica *rep, int nsteps) {
  /* Molecules::ExecuteSteps (src/integrator.cxx:708-723): the velocity-scaling
     thermostat (tconstant 2) rescales before every step */
  for (int s = 0; s < nsteps; s++) {
    if (TMODE(sys) == 2) {
      orc_velocity_scaling(sys, rep);
      orc_ang_velocity_scaling(sys, rep);
    }
    orc_step(sys, rep);
  }
  orc_calc_properties(sys, rep);
}

void orc_initialize_property(const orc_system *sys, orc_replica *rep) {
  orc_force(sys, rep);
  rep->gkT = 6.0 * (double)sys->nmol * rep->T;
  orc_calc_properties(sys, rep);
  rep->H0 = rep->tot;
  rep->ham = rep->tot - rep->H0;
}

static void kill_angular_momentum_in_tube(const orc_system *sys, orc_replica *rep) {
  /* src/molecules.cxx:189-210 */
  double mom = 0., msum = 0.;
  for (int i = 0; i < sys->nmol; i++) {
    double r[3], v[3];
    for (int d = 0; d < 3; d++) r[d] = (rep->r[3 * i + d] - 0.5) * rep->L[d];
    for (int d = 0; d < 3; d++) v[d] = rep->v[3 * i + d] / (rep->L[d] * rep->s);
    const double m = rep->m[i];
    mom += m * (r[0] * v[1] - r[1] * v[0]);
    msum += m;
  }
  mom /= msum;
  for (int i = 0; i < sys->nmol; i++) {
    double r[3];
    for (int d = 0; d < 3; d++) r[d] = (rep->r[3 * i + d] - 0.5) * rep->L[d];
    const double r02 = r[0] * r[0] + r[1] * r[1];
    if (r02 > 1.0) {
      rep->v[3 * i + 0] += mom * r[1] / r02 * rep->L[0] * rep->s;
      rep->v[3 * i + 1] -= mom * r[0] / r02 * rep->L[1] * rep->s;
    }
  }
}

void orc_kill_momentum(const orc_system *sys, orc_replica *rep) {
  /* src/molecules.cxx:168-187 */
  double sum[3] = {0, 0, 0}, m = 0.;
  for (int i = 0; i < sys->nmol; i++) {
    for (int d = 0; d < 3; d++) sum[d] += rep->v[3 * i + d] * rep->m[i];
    m += rep->m[i];
  }
  for (int d = 0; d < 3; d++) sum[d] /= m;
  if (sys->confined == 1) {
    for (int i = 0; i < sys->nmol; i++) rep->v[3 * i + 2] -= sum[2];
    kill_angular_momentum_in_tube(sys, rep);
  } else if (sys->confined == 2) {
    for (int i = 0; i < sys->nmol; i++) {
      rep->v[3 * i + 0] -= sum[0];
      rep->v[3 * i + 1] -= sum[1];
    }
  } else {
    for (int i = 0; i < sys->nmol; i++)
      for (int d = 0; d < 3; d++) rep->v[3 * i + d] -= sum[d];
  }
}

void orc_velocity_scaling(const orc_system *sys, orc_replica *rep) {
  /* src/molecules.cxx:261-273 */
  double k[3];
  translational_energy(sys, rep, k);
  const double tra = k[0] + k[1] + k[2];
  if (tra == 0.) return;
  const double coef = sqrt(1.5 * sys->nmol * rep->T / tra);
  for (int i = 0; i < 3 * sys->nmol; i++) rep->v[i] *= coef;
  orc_kill_momentum(sys, rep);
  if (sys->confined == 1) kill_angular_momentum_in_tube(sys, rep);
  rep->s = 1.0;
  rep->Ps = 0.0;
  rep->Pv[0] = rep->Pv[1] = rep->Pv[2] = 0.0;
}

void orc_ang_velocity_scaling(const orc_system *sys, orc_replica *rep) {
  /* src/molecules.cxx:296-311 */
  const double rot = rotational_energy(sys, rep);
  if (rot == 0.) return;
  const double coef = sqrt(1.5 * sys->nmol * rep->T / rot);
  for (int i = 0; i < 4 * sys->nmol; i++) rep->p[i] *= coef;
}

void orc_change_temperature(const orc_system *sys, orc_replica *rep, double Tnew) {
  /* src/molecules.h:333-353 */
  const double coef = sqrt(Tnew / rep->T);
  for (int i = 0; i < 3 * sys->nmol; i++) rep->v[i] *= coef / rep->s;
  for (int i = 0; i < 4 * sys->nmol; i++) rep->p[i] *= coef / rep->s;
  rep->Ps *= coef;
  if (sys->pconstant == 1) rep->Pv[0] *= coef * rep->s;
  if (sys->pconstant == 2) rep->Pv[2] *= coef * rep->s;
  if (sys->pconstant == 3) {
    rep->Pv[0] *= coef * rep->s;
    rep->Pv[1] *= coef * rep->s;
  }
  rep->T = Tnew;
  rep->gkT = 6.0 * (double)sys->nmol * rep->T;
  rep->s = 1.0;
}

void orc_apply_condition(const orc_system *sys, orc_replica *rep, double Tnew, double Pnew) {
  orc_change_temperature(sys, rep, Tnew);
  orc_kill_momentum(sys, rep);
  rep->P = Pnew;
  orc_calc_properties(sys, rep);
  rep->H0 = rep->tot;
  rep->ham = 0.0;
}

/* ---- exchange ---- */
void orc_exchange_lists(int dim_temp, int dim_press, int *lists, int len[4]) {
  /* ExchangeList::ExchangeList, src/remdinfo.cxx:54-125 */
  const int cap = dim_temp * dim_press / 2;
  int *l0 = lists, *l1 = lists + 2 * cap, *l2 = lists + 4 * cap, *l3 = lists + 6 * cap;
  int c = 0;
  for (int j = 0; j < dim_press; ++j)
    for (int i = 0; i < dim_temp / 2; ++i) {
      l0[2 * c] = 2 * i + j * dim_temp;
      l0[2 * c + 1] = 2 * i + 1 + j * dim_temp;
      c++;
    }
  len[0] = c;
  c = 0;
  for (int j = 0; j < dim_press / 2; ++j)
    for (int i = 0; i < dim_temp; ++i) {
      l1[2 * c] = i + 2 * j * dim_temp;
      l1[2 * c + 1] = i + (2 * j + 1) * dim_temp;
      c++;
    }
  len[1] = c;
  c = 0;
  for (int j = 0; j < dim_press; ++j)
    for (int i = 0; i < dim_temp / 2 - (dim_temp + 1) % 2; ++i) {
      l2[2 * c] = 2 * i + j * dim_temp + 1;
      l2[2 * c + 1] = 2 * i + 1 + j * dim_temp + 1;
      c++;
    }
  len[2] = c;
  c = 0;
  for (int j = 0; j < dim_press / 2 - (dim_press + 1) % 2; ++j)
    for (int i = 0; i < dim_temp; ++i) {
      l3[2 * c] = i + (2 * j + 1) * dim_temp;
      l3[2 * c + 1] = i + (2 * j + 2) * dim_temp;
      c++;
    }
  len[3] = c;
}

void orc_conditions_geometrical(int dim_temp, int dim_press, double tmin_K, double tmax_K,
                                double pmin_Pa, double pmax_Pa, double *T, double *P) {
  /* REMDInfo ctor (src/remdinfo.cxx:167-170) + SetConditionGeometrical (348-359) */
  const double temperature_max = tmax_K / orc_unit_temp();
  const double temperature_min = tmin_K / orc_unit_temp();
  const double pressure_max = pmax_Pa / orc_unit_press();
  const double pressure_min = pmin_Pa / orc_unit_press();
  const double t = (dim_temp == 1) ? 1.0 : powf((float)(temperature_max / temperature_min), (float)(1. / (double)(dim_temp - 1)));
  const double p = (dim_press == 1) ? 0.0 : ((pressure_max - pressure_min) / (double)(dim_press - 1));
  for (int j = 0; j < dim_press; ++j)
    for (int i = 0; i < dim_temp; ++i) {
      const int ind = i + j * dim_temp;
      T[ind] = temperature_min * powf((float)t, (float)i);
      P[ind] = pressure_min + p * j;
    }
}

int orc_replica_exchange(int ntemp, int npress, int pconstant, long step, int *index,
                         double *temperature, double *pressure, const double *pot,
                         const double *vol, const double *u, int *accepted,
                         unsigned char *is_exchanged) {
  /* REMD::ReplicaExchange + CalcExchangeProb, src/remd.cxx:467-538;
   * ExchangeAccepted/Rejected, src/remdinfo.h:345-359 */
  const int cap = ntemp * npress / 2;
  int *lists = (int *)malloc(sizeof(int) * 8 * (cap > 0 ? cap : 1));
  int len[4];
  orc_exchange_lists(ntemp, npress, lists, len);
  const int n = ntemp * npress;
  for (int i = 0; i < n; i++) is_exchanged[i] = 0;
  const int ec_type = (int)(step % 4);
  const int *l = lists + 2 * cap * ec_type;
  for (int i = 0; i < len[ec_type]; ++i) {
    const int a = l[2 * i], b = l[2 * i + 1];
    const int ind1 = index[a], ind2 = index[b];
    const double beta1 = 1. / temperature[ind1];
    const double beta2 = 1. / temperature[ind2];
    double delta = (beta2 - beta1) * (pot[ind1] - pot[ind2]);
    if (pconstant > 0) delta += (beta2 * pressure[ind2] - beta1 * pressure[ind1]) * (vol[ind1] - vol[ind2]);
    const double prob = exp(-delta);
    if (prob > u[i]) {
      is_exchanged[index[a]] = 1;
      is_exchanged[index[b]] = 1;
      double tmp = temperature[index[a]];
      temperature[index[a]] = temperature[index[b]];
      temperature[index[b]] = tmp;
      tmp = pressure[index[a]];
      pressure[index[a]] = pressure[index[b]];
      pressure[index[b]] = tmp;
      const int ti = index[a];
      index[a] = index[b];
      index[b] = ti;
      accepted[i] = 1;
    } else {
      is_exchanged[index[a]] = 0;
      is_exchanged[index[b]] = 0;
      accepted[i] = 0;
    }
  }
  free(lists);
  return len[ec_type];
}
