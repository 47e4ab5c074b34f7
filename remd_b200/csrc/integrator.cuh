// integrator.cuh -- the Nose-Poincare thermostat / Andersen barostat quaternion
// integrator of the reference (src/integrator.cxx:132-706), FP64, split into
// the per-replica scalar chain (run by one thread and broadcast) and the
// per-molecule free-rotor / drift / kick operators (one thread per molecule).
//
// Operation order follows the reference CPU code so the FP64 results agree
// with it to rounding; confined=2 (slit) barostat terms follow the reference
// GPU kernel (src/remdgpu.cu:2083-2120, 2537-2545, 2803-2809), since the
// reference CPU slit path does not run (src/force_calculator.cxx:1525, 1556-1561).
#pragma once
#include "engine_types.cuh"

namespace remd {

__host__ __device__ inline double volume(const RepConst& c, const RepState& st) {
  // Molecules::GetVolume / GetBottomArea, src/molecules.h:357-376
  if (c.confined == 1) return c.bottom_area * st.L[2];
  if (c.confined == 2) return st.L[0] * st.L[1] * c.slit_width;
  return st.L[0] * st.L[1] * st.L[2];
}

// D6: thermostat half step, src/integrator.cxx:634-644
__device__ inline void d6(const RepConst& c, RepState& st) {
  if (c.tconstant == 1) {
    const double tmp = 1.0 + (st.Ps / (2.0 * c.Q) * c.dthalf);
    st.s *= tmp * tmp;
    st.Ps /= tmp;
  }
}

// D5 scalar part (src/integrator.cxx:583-600; slit src/remdgpu.cu:2537-2545)
__device__ inline void d5_scalar(const RepConst& c, RepState& st, double pot, const double* vir) {
  const double dthalf = c.dthalf;
  if (c.tconstant == 1) {
    st.Ps -= pot * dthalf;
    if (c.pconstant > 0) st.Ps -= (st.P * volume(c, st)) * dthalf;
  }
  if (c.pconstant == 1)
    st.Pv[0] += ((vir[0] + vir[1] + vir[2]) / (3.0 * st.L[0] * st.L[1] * st.L[2]) - st.P) * st.s * dthalf;
  if (c.pconstant == 2)
    st.Pv[2] += st.s * (vir[2] / st.L[2] - st.P * c.bottom_area) * dthalf;
  if (c.pconstant == 3) {
    const double zlen = (c.confined == 2) ? c.wall_length_param : st.L[2];
    st.Pv[0] += st.s * (vir[0] / st.L[0] - st.P * st.L[1] * zlen) * dthalf;
    st.Pv[1] += st.s * (vir[1] / st.L[1] - st.P * st.L[0] * zlen) * dthalf;
  }
}

// D4: barostat half step, src/integrator.cxx:604-632 (slit: src/remdgpu.cu:2096-2115)
__device__ inline void d4(const RepConst& c, RepState& st) {
  const double dthalf = c.dthalf;
  if (c.pconstant == 1) {
    if (c.tconstant == 1) st.Ps -= st.Pv[0] * st.Pv[0] / c.W * dthalf;
    const double V = volume(c, st);
    // the reference takes the cube root in single precision (powf(float, float),
    // src/integrator.cxx:614); evaluated here in double and rounded once to
    // float, i.e. the correctly rounded single-precision result
    const float xf = (float)(V + st.Pv[0] * st.s / c.W * dthalf);
    const double Ln = (double)(float)pow((double)xf, (double)(float)(1. / 3.));
    st.L[0] = st.L[1] = st.L[2] = Ln;
  }
  if (c.pconstant == 2) {
    if (c.tconstant == 1) st.Ps -= 0.5 * st.Pv[2] * st.Pv[2] / c.W * dthalf;
    st.L[2] += st.s * st.Pv[2] / c.W * dthalf;
  }
  if (c.pconstant == 3) {
    const double bw = 0.5 / c.W;
    if (c.tconstant == 1) st.Ps -= (st.Pv[0] * st.Pv[0] + st.Pv[1] * st.Pv[1]) * bw * dthalf;
    st.L[0] += st.s * st.Pv[0] * bw * c.dt;
    st.L[1] += st.s * st.Pv[1] * bw * c.dt;
  }
}

// D3D2D1D2D3_PsPv, src/integrator.cxx:132-172
__device__ inline void pspv(const RepConst& c, RepState& st, double* sum_Pv, double sum_Ps) {
  const bool needPv = (c.pconstant > 0 || c.tconstant == 1);
  if (needPv)
    for (int d = 0; d < 3; d++) sum_Pv[d] /= st.L[d] * st.L[d] * st.s * st.s;
  const double sPv = sum_Pv[0] + sum_Pv[1] + sum_Pv[2];
  if (c.pconstant == 1) st.Pv[0] += st.s * sPv / (volume(c, st) * 3.0) * c.dthalf;
  if (c.pconstant == 2) st.Pv[2] += st.s * sum_Pv[2] / st.L[2] * c.dthalf;
  if (c.pconstant == 3) {
    st.Pv[0] += st.s * sum_Pv[0] / st.L[0] * c.dthalf;
    st.Pv[1] += st.s * sum_Pv[1] / st.L[1] * c.dthalf;
  }
  if (c.tconstant == 1)
    st.Ps += (0.25 * sPv + 2.0 * sum_Ps - (1.0 + log(st.s)) * st.gkT + st.H0) * c.dt;
}

// body_to_space / space_to_body, src/rotation.h:146-187
__host__ __device__ inline void body_to_space(const double* a, const double* v, double* o) {
  const double a0sq = a[0] * a[0], a1sq = a[1] * a[1], a2sq = a[2] * a[2], a3sq = a[3] * a[3];
  const double a01 = a[0] * a[1], a02 = a[0] * a[2], a03 = a[0] * a[3];
  const double a12 = a[1] * a[2], a13 = a[1] * a[3], a23 = a[2] * a[3];
  o[0] = (a0sq + a1sq - a2sq - a3sq) * v[0] + 2. * (a12 - a03) * v[1] + 2. * (a13 + a02) * v[2];
  o[1] = 2. * (a12 + a03) * v[0] + (a0sq - a1sq + a2sq - a3sq) * v[1] + 2. * (a23 - a01) * v[2];
  o[2] = 2. * (a13 - a02) * v[0] + 2. * (a23 + a01) * v[1] + (a0sq - a1sq - a2sq + a3sq) * v[2];
}

__host__ __device__ inline void space_to_body(const double* a, const double* v, double* o) {
  const double a0sq = a[0] * a[0], a1sq = a[1] * a[1], a2sq = a[2] * a[2], a3sq = a[3] * a[3];
  const double a01 = a[0] * a[1], a02 = a[0] * a[2], a03 = a[0] * a[3];
  const double a12 = a[1] * a[2], a13 = a[1] * a[3], a23 = a[2] * a[3];
  o[0] = (a0sq + a1sq - a2sq - a3sq) * v[0] + 2. * (a12 + a03) * v[1] + 2. * (a13 - a02) * v[2];
  o[1] = 2. * (a12 - a03) * v[0] + (a0sq - a1sq + a2sq - a3sq) * v[1] + 2. * (a23 + a01) * v[2];
  o[2] = 2. * (a13 + a02) * v[0] + 2. * (a23 - a01) * v[1] + (a0sq - a1sq - a2sq + a3sq) * v[2];
}

// The free-rotor sub-step about body axis `axis` (D1: x, D2: y, D3: z),
// src/integrator.cxx:467-563: (q,p) -> (q cos + P_k(q) sin, p cos + P_k(p) sin).
__device__ inline double rotate(double* q, double* p, int axis, double Ik, double coef_xi, double h) {
  double Pq[4], Pp[4];
  if (axis == 1) {
    Pq[0] = -q[1]; Pq[1] = q[0]; Pq[2] = q[3]; Pq[3] = -q[2];
    Pp[0] = -p[1]; Pp[1] = p[0]; Pp[2] = p[3]; Pp[3] = -p[2];
  } else if (axis == 2) {
    Pq[0] = -q[2]; Pq[1] = -q[3]; Pq[2] = q[0]; Pq[3] = q[1];
    Pp[0] = -p[2]; Pp[1] = -p[3]; Pp[2] = p[0]; Pp[3] = p[1];
  } else {
    Pq[0] = -q[3]; Pq[1] = q[2]; Pq[2] = -q[1]; Pq[3] = q[0];
    Pp[0] = -p[3]; Pp[1] = p[2]; Pp[2] = -p[1]; Pp[3] = p[0];
  }
  const double xi = (((p[0] * Pq[0] + p[1] * Pq[1]) + p[2] * Pq[2]) + p[3] * Pq[3]) * coef_xi / Ik;
  double sn, cs;
  sincos(xi * h, &sn, &cs);
  for (int k = 0; k < 4; k++) q[k] = q[k] * cs + Pq[k] * sn;
  for (int k = 0; k < 4; k++) p[k] = p[k] * cs + Pp[k] * sn;
  return xi;
}

// D5 per-molecule kick (src/integrator.cxx:572-582): v += f*coef_v/m, p += S(q) n coef_p
__device__ inline void kick(double* v, double* p, const double* q, const double* f, const double* n,
                            const double* coef_v, double coef_p, double m) {
  for (int d = 0; d < 3; d++) v[d] += f[d] * coef_v[d] / m;
  const double Sn0 = ((q[0] * n[0] + (-q[1]) * n[1]) + (-q[2]) * n[2]) + (-q[3]) * n[3];
  const double Sn1 = ((q[1] * n[0] + q[0] * n[1]) + (-q[3]) * n[2]) + q[2] * n[3];
  const double Sn2 = ((q[2] * n[0] + q[3] * n[1]) + q[0] * n[2]) + (-q[1]) * n[3];
  const double Sn3 = ((q[3] * n[0] + (-q[2]) * n[1]) + q[1] * n[2]) + q[0] * n[3];
  p[0] += Sn0 * coef_p;
  p[1] += Sn1 * coef_p;
  p[2] += Sn2 * coef_p;
  p[3] += Sn3 * coef_p;
}

// Per-molecule kinetic terms of CalcProperties (src/molecules.cxx:631-657):
// tra3 += (v*v)*m per dimension; rot += I*xi*xi*2 with xi = p.P_k(q) * (1/I)*coef.
__device__ inline double rot_energy(const double* q, const double* p, const double* I, double s) {
  const double coef = 0.25 / s;
  double xi[3];
  xi[0] = ((p[0] * (-q[1]) + p[1] * q[0]) + p[2] * q[3]) + p[3] * (-q[2]);
  xi[1] = ((p[0] * (-q[2]) + p[1] * (-q[3])) + p[2] * q[0]) + p[3] * q[1];
  xi[2] = ((p[0] * (-q[3]) + p[1] * q[2]) + p[2] * (-q[1])) + p[3] * q[0];
  double r = 0.0;
  for (int k = 0; k < 3; k++) {
    const double x = xi[k] * ((1.0 / I[k]) * coef);
    r += I[k] * x * x * 2.0;
  }
  return r;
}

}  // namespace remd
