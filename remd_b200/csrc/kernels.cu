// kernels.cu -- device code of the B200 REMD engine.  See kernels.cuh for the
// step decomposition and engine_types.cuh for the data layout.
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <type_traits>

#include "integrator.cuh"
#include "kernels.cuh"

namespace cg = cooperative_groups;

namespace remd {

constexpr int kRepThreads = 256;   // threads of the per-replica kernels
constexpr int kBitmapMaxWords = 64; // list-rebuild bitmap window: 2048 molecules per pass
constexpr int kCellMinPrune = 4;    // cut a replica into cells when they prune at least 4x
constexpr int kListLanes = 4;       // lanes per molecule in the FP32 list kernel (adjacent in a warp)

int pack_stride(int nsite, int prec) {
  if (prec == kF32) return ((3 + 3 * nsite) + 3) / 4 * 4;   // words, 16-B multiple
  return ((3 + 3 * nsite) + 1) / 2 * 2;                      // doubles, 16-B multiple
}

// ------------------------------------------------------------------ reductions
template <int K>
__device__ inline void block_sum(double* v, double* sm) {
  // deterministic: fixed shuffle tree, then warp partials summed in warp order
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < K; k++)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  __syncthreads();
  if (lane == 0)
    for (int k = 0; k < K; k++) sm[warp * K + k] = v[k];
  __syncthreads();
  for (int k = 0; k < K; k++) {
    double t = 0.0;
    for (int w = 0; w < nw; w++) t += sm[w * K + k];
    v[k] = t;
  }
  __syncthreads();
}

__device__ inline double block_max(double v, double* sm) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  __syncthreads();
  if (lane == 0) sm[warp] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < nw; w++) t = fmax(t, sm[w]);
  __syncthreads();
  return t;
}

// Deterministic warp reductions (fixed xor tree; lane 0's value is used).
template <int K>
__device__ inline void warp_sum(double* v) {
#pragma unroll
  for (int k = 0; k < K; k++)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
}

__device__ inline double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Sum of the force partials of replica c (ordered pairs -> halved like
// ForceCalculator::Switching, src/force_calculator.cxx:775-778).  Called by
// all 32 lanes of one warp: lane l sums records l, l+32, ..., then a butterfly
// over the lanes.  Every lane ends with the same bits (the two partners of a
// butterfly step add the same two numbers) and the order depends only on the
// replica's record count, so every kernel that needs the sums gets identical
// values.  One warp loads all records at once instead of one thread walking
// them: the per-replica scalar chains of the step kernels start sooner.
struct P2Sum {
  double lj, clmb, wall, vir[3];
};
__device__ inline P2Sum reduce_part2(const DevPtrs& d, const RepConst& c) {
  double v[6] = {0, 0, 0, 0, 0, 0};
  for (int t = c.warp_off + (threadIdx.x & 31); t < c.warp_off + c.nwarp; t += 32) {
    const Part2 p = d.part2[t];
    v[0] += p.lj; v[1] += p.clmb; v[2] += p.wall;
    v[3] += p.vir[0]; v[4] += p.vir[1]; v[5] += p.vir[2];
  }
  warp_sum<6>(v);
  P2Sum e;
  e.lj = v[0] * 0.5;
  e.clmb = v[1] * 0.5;
  e.wall = v[2];
  e.vir[0] = v[3] * 0.5; e.vir[1] = v[4] * 0.5; e.vir[2] = v[5] * 0.5;
  return e;
}

// Programmatic dependent launch of the MD-step kernels (launch_integrate_prec,
// launch_force): where a step's tile grid is smaller than the GPU, each is
// launched allowed to start while the kernel before it on its stream is still
// running.  Its blocks first wait for that kernel's completion and memory
// (griddepcontrol.wait, which returns at once when there is no such kernel or
// the launch was a plain one), then let the next kernel be scheduled.  A step
// kernel thus reads nothing of its predecessor early; what overlaps is the
// next launch's scheduling with this kernel's last wave.
__device__ __forceinline__ void step_kernel_entry() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Difference of two fixed-point box fractions with 32-bit wraparound: the
// minimum-image separation in units of L / 2^32 (defined via unsigned arithmetic).
__device__ __forceinline__ int wrap_diff(int a, int b) { return (int)((unsigned)a - (unsigned)b); }

// ------------------------------------------------------------------ force records
__device__ inline int fix_coord(double r) {
  // box fraction in [0,1) -> (r-0.5)*2^32 as a wrapping int32
  return (int)(unsigned int)(long long)llrint((r - 0.5) * kFix);
}

__device__ inline void write_pack(const DevPtrs& d, const RepConst& c, int prec, int li,
                                  const double* r, const double* q) {
  const int ns = c.nsite;
  if (prec == kF32) {
    uint32_t* w = reinterpret_cast<uint32_t*>(d.pack) + c.pack_off + (long long)li * c.pack_stride;
    uint32_t buf[20];
    for (int k = 0; k < 20; k++) buf[k] = 0u;
    buf[0] = (uint32_t)fix_coord(r[0]);
    buf[1] = (uint32_t)fix_coord(r[1]);
    buf[2] = (uint32_t)fix_coord(r[2]);
    for (int k = 0; k < ns; k++) {
      double o[3];
      body_to_space(q, c.body[k], o);
      for (int x = 0; x < 3; x++) buf[3 + 3 * k + x] = __float_as_uint((float)o[x]);
    }
    uint4* w4 = reinterpret_cast<uint4*>(w);
    for (int k = 0; k < c.pack_stride / 4; k++)
      w4[k] = make_uint4(buf[4 * k], buf[4 * k + 1], buf[4 * k + 2], buf[4 * k + 3]);
    d.com[c.mol_off + li] = make_int4((int)buf[0], (int)buf[1], (int)buf[2], 0);
  } else {
    double* w = reinterpret_cast<double*>(d.pack) + c.pack_off + (long long)li * c.pack_stride;
    w[0] = r[0]; w[1] = r[1]; w[2] = r[2];
    for (int k = 0; k < ns; k++) {
      double o[3];
      body_to_space(q, c.body[k], o);
      for (int x = 0; x < 3; x++) w[3 + 3 * k + x] = o[x];
    }
    // fixed-point centre: the cell of the molecule at the next list build
    d.com[c.mol_off + li] = make_int4(fix_coord(r[0]), fix_coord(r[1]), fix_coord(r[2]), 0);
  }
}

__global__ void k_pack(DevPtrs d, int prec) {
  const Tile t = d.tiles[blockIdx.x];
  const RepConst& c = d.rc[t.rep];
  const int i = threadIdx.x;
  if (i < t.count) {
    const int li = t.start + i;
    const int g = c.mol_off + li;
    double r[3], q[4];
    for (int x = 0; x < 3; x++) r[x] = d.r[x * d.N + g];
    for (int x = 0; x < 4; x++) q[x] = d.q[x * d.N + g];
    write_pack(d, c, prec, li, r, q);
  }
  if (i == 0) {
    const double nan = __longlong_as_double(0x7ff8000000000000ll);
    d.Lbuild[3 * blockIdx.x] = nan;   // lists must be rebuilt
  }
}

// ------------------------------------------------------------------ integrate
struct StepCoef {
  double coef_v_a[3], coef_p_a;   // end-of-previous-step kick
  double coef_v_c[3], coef_p_c;   // this step's kick
  double coef_xi, cxi1, coef_r[3];
  double Lb[3];
};

template <bool MID>
__global__ void __launch_bounds__(128, 7) k_integrate(DevPtrs d, const RepState* __restrict__ X,
                                                   RepState* __restrict__ Y, int prec) {
  step_kernel_entry();
  __shared__ StepCoef sc;
  const int tix = d.tile0 + blockIdx.x;   // this launch's tile range
  const Tile t = d.tiles[tix];
  const RepConst& c = d.rc[t.rep];
  P2Sum e;
  if (threadIdx.x < 32) e = reduce_part2(d, c);
  if (threadIdx.x == 0) {
    RepState st = X[t.rep];
    const double pot = e.lj + e.clmb + e.wall;
    if (MID) {   // D5 (scalar) + D6 closing the previous step
      for (int x = 0; x < 3; x++) sc.coef_v_a[x] = st.L[x] * st.s * c.dthalf;
      sc.coef_p_a = 2.0 * st.s * c.dthalf;
      d5_scalar(c, st, pot, e.vir);
      d6(c, st);
    }
    d6(c, st);   // D6 opening this step
    for (int x = 0; x < 3; x++) sc.coef_v_c[x] = st.L[x] * st.s * c.dthalf;
    sc.coef_p_c = 2.0 * st.s * c.dthalf;
    d5_scalar(c, st, pot, e.vir);
    d4(c, st);
    sc.coef_xi = 0.25 / st.s;
    const double si = 1.0 / st.s;
    sc.cxi1 = 0.25 * si;
    for (int x = 0; x < 3; x++) {
      const double Li = 1.0 / st.L[x];
      sc.coef_r[x] = Li * Li * si * c.dt;
    }
    for (int x = 0; x < 3; x++) sc.Lb[x] = d.Lbuild[3 * tix + x];
    if (tix == c.tile_off) Y[t.rep] = st;
  }
  __syncthreads();
  const int i = threadIdx.x;
  double acc[4] = {0, 0, 0, 0};
  double disp = 0.0;
  if (i < t.count) {
    const int li = t.start + i;
    const int g = c.mol_off + li;
    const int N = d.N;
    double r[3], v[3], q[4], p[4], f[3], n[4];
    for (int x = 0; x < 3; x++) { r[x] = d.r[x * N + g]; v[x] = d.v[x * N + g]; f[x] = d.f[x * N + g]; }
    for (int x = 0; x < 4; x++) { q[x] = d.q[x * N + g]; p[x] = d.p[x * N + g]; n[x] = d.n[x * N + g]; }
    const double m = c.mass;
    if (MID) kick(v, p, q, f, n, sc.coef_v_a, sc.coef_p_a, m);
    kick(v, p, q, f, n, sc.coef_v_c, sc.coef_p_c, m);
    const bool T1 = (c.tconstant == 1);
    double sPs = 0.0;
    double xi = rotate(q, p, 3, c.I[2], sc.coef_xi, c.dthalf);
    if (T1) sPs += 0.5 * xi * xi * c.I[2];
    xi = rotate(q, p, 2, c.I[1], sc.coef_xi, c.dthalf);
    if (T1) sPs += 0.5 * xi * xi * c.I[1];
    for (int x = 0; x < 3; x++) {
      r[x] += v[x] * sc.coef_r[x];
      if (r[x] < 0.0) r[x] += 1.0;
      if (r[x] >= 1.0) r[x] -= 1.0;
    }
    xi = rotate(q, p, 1, c.I[0], sc.cxi1, c.dt);
    if (c.pconstant > 0 || T1)
      for (int x = 0; x < 3; x++) acc[x] = 2.0 * m * v[x] * v[x];
    if (T1) sPs += xi * xi * c.I[0];
    xi = rotate(q, p, 2, c.I[1], sc.coef_xi, c.dthalf);
    if (T1) sPs += 0.5 * xi * xi * c.I[1];
    xi = rotate(q, p, 3, c.I[2], sc.coef_xi, c.dthalf);
    if (T1) sPs += 0.5 * xi * xi * c.I[2];
    acc[3] = sPs;
    for (int x = 0; x < 3; x++) { d.r[x * N + g] = r[x]; d.v[x * N + g] = v[x]; }
    for (int x = 0; x < 4; x++) { d.q[x * N + g] = q[x]; d.p[x * N + g] = p[x]; }
    write_pack(d, c, prec, li, r, q);
    // displacement since the last neighbour-list build, in the build box
    const int4 ref = d.ref_com[g];
    const int fx = fix_coord(r[0]), fy = fix_coord(r[1]), fz = fix_coord(r[2]);
    const double dx = (double)wrap_diff(fx, ref.x) * kFixInv * sc.Lb[0];
    const double dy = (double)wrap_diff(fy, ref.y) * kFixInv * sc.Lb[1];
    const double dz = (double)wrap_diff(fz, ref.z) * kFixInv * sc.Lb[2];
    disp = sqrt(dx * dx + dy * dy + dz * dz);
    if (!(disp == disp)) disp = 1e30;   // NaN box: force a rebuild
  }
  warp_sum<4>(acc);
  disp = warp_max(disp);
  const int w = (t.start + threadIdx.x) >> 5;   // 32-molecule unit of the replica
  if ((threadIdx.x & 31) == 0 && w < c.nwarp) {
    Part1 pt;
    pt.sum_Pv[0] = acc[0]; pt.sum_Pv[1] = acc[1]; pt.sum_Pv[2] = acc[2];
    pt.sum_Ps = acc[3];
    pt.disp = disp;
    d.part1[c.warp_off + w] = pt;
  }
}

// ------------------------------------------------------------------ force
// Cell of a fixed-point box fraction x = (r - 1/2) 2^32 on an n-cell axis:
// floor(r n), exact (r 2^32 = x + 2^31 as an unsigned word).
__device__ __forceinline__ int cell_coord(int x, int n) {
  const unsigned u = (unsigned)x + 0x80000000u;
  return (int)(((unsigned long long)u * (unsigned)n) >> 32);
}

// Radius the list build tests (FP32 form): rcut + skin widened by the
// truncation error of its FP32 test, sqrt(3) L_max 2^-16, and a relative 1e-5.
// The FP64 form's test radius, rcut + skin, is below it.
__device__ inline double list_test_radius(const RepConst& c, const double* L) {
  const double lmax = fmax(fmax(L[0], L[1]), L[2]);
  return (c.rc + c.skin + 1.7320508075688772 * lmax * (1.0 / 65536.0)) * (1.0 + 1e-5);
}

// Cells per dimension: as many as fit at least the test radius wide, so that
// every pair the list build keeps lies in neighbouring cells; a dimension with
// fewer than three such cells is not cut (one cell), and the grid is coarsened
// along its longest axis until it has at most kMaxCells cells.
__device__ inline CellGrid cell_grid(const RepConst& c, const double* L) {
  // a cell is wider than any component the FP32 test can keep (its truncated
  // differences err by less than L 2^-16 per component), so the lists equal
  // those of a test against every molecule of the replica
  const double lmax = fmax(fmax(L[0], L[1]), L[2]);
  const double rw = list_test_radius(c, L) + 2.0 * lmax * (1.0 / 65536.0);
  int n[3];
  for (int x = 0; x < 3; x++) {
    const double q = L[x] / rw;
    n[x] = (q >= 3.0) ? (int)fmin(floor(q), (double)kMaxCells) : 1;   // NaN -> 1
  }
  while ((long long)n[0] * n[1] * n[2] > kMaxCells) {
    const int m = (n[0] >= n[1] && n[0] >= n[2]) ? 0 : (n[1] >= n[2] ? 1 : 2);
    n[m] = (n[m] - 1 >= 3) ? n[m] - 1 : 1;
  }
  // a candidate from the cells costs several times one of the all-molecule scan
  // (gathered, per lane, versus a shared-memory broadcast): cut the box only
  // where the neighbouring cells hold at most 1/kCellMinPrune of the replica
  const int stencil = (n[0] > 1 ? 3 : 1) * (n[1] > 1 ? 3 : 1) * (n[2] > 1 ? 3 : 1);
  if ((long long)stencil * kCellMinPrune > (long long)n[0] * n[1] * n[2]) n[0] = n[1] = n[2] = 1;
  CellGrid g;
  g.nx = n[0]; g.ny = n[1]; g.nz = n[2];
  g.rebuild = 1;
  return g;
}

// The kListLanes bits of a warp ballot that belong to this lane's molecule.
__device__ __forceinline__ unsigned group_bits(unsigned ballot, int lane) {
  return (ballot >> (lane & ~(kListLanes - 1))) & ((1u << kListLanes) - 1u);
}

__device__ inline int cell_of(const int4 x, const CellGrid& g) {
  return (cell_coord(x.z, g.nz) * g.ny + cell_coord(x.y, g.ny)) * g.nx + cell_coord(x.x, g.nx);
}

// Per-replica head of a force step, one block per replica of the launch:
//  * warp 0 sums the integrate kernel's partials (lane-strided, then a
//    butterfly, so the order depends only on the replica's record count) and
//    lane 0 runs PsPv and D4 (src/integrator.cxx:132-172, 604-632), writes the
//    replica's scalars to Xout and decides whether its neighbour lists must be
//    rebuilt: pairs now within rc were within rc + skin at the build if
//    2 max|displacement| + rc (max_d Lbuild_d / L_d - 1) <= skin;
//  * when they must, the block counting-sorts the replica's molecules by cell
//    (cell_grid) into cell_start / cell_com; k_force_lists then tests each
//    molecule against the molecules of its 27 (tube: 3, slit: 9) neighbouring
//    cells only.  The order inside a cell is arbitrary: the lists are emitted
//    in ascending j from a bitmap (build_lists), so they do not depend on it.
// This replaces the reference's per-replica z-sort of the molecules
// (sort, src/sort.cu:373-459; quicksort_key, src/quicksort.cu:214-276).
template <bool FORCE_ONLY>
__global__ void __launch_bounds__(kRepThreads) k_replica_head(DevPtrs d, const RepState* __restrict__ Yin,
                                                              RepState* __restrict__ Xout) {
  step_kernel_entry();
  __shared__ int cnt[kMaxCells];
  __shared__ int wsum[kRepThreads / 32];
  __shared__ CellGrid grid;
  const int rep = d.rep0 + blockIdx.x;
  const RepConst& c = d.rc[rep];
  if (threadIdx.x < 32) {
    double v[4] = {0, 0, 0, 0}, disp = 0.0;
    if (!FORCE_ONLY) {
      for (int k = c.warp_off + threadIdx.x; k < c.warp_off + c.nwarp; k += 32) {
        const Part1 p = d.part1[k];
        v[0] += p.sum_Pv[0]; v[1] += p.sum_Pv[1]; v[2] += p.sum_Pv[2];
        v[3] += p.sum_Ps;
        disp = fmax(disp, p.disp);
      }
      warp_sum<4>(v);
      disp = warp_max(disp);
    }
    if (threadIdx.x == 0) {
      RepState st = Yin[rep];
      int rb = 1;
      if (!FORCE_ONLY) {
        double sPv[3] = {v[0], v[1], v[2]};
        pspv(c, st, sPv, v[3]);
        d4(c, st);
        const int tix = c.tile_off;   // every tile of a replica holds the same build box
        const double lb0 = d.Lbuild[3 * tix], lb1 = d.Lbuild[3 * tix + 1], lb2 = d.Lbuild[3 * tix + 2];
        rb = !(lb0 == lb0);
        if (!rb) {
          const double lam = fmax(fmax(lb0 / st.L[0], lb1 / st.L[1]), lb2 / st.L[2]);
          rb = (2.0 * disp + c.rc * (lam - 1.0) > c.skin);
        }
      }
      Xout[rep] = st;   // FORCE_ONLY launches pass Xout == Yin: unchanged there
      CellGrid g = cell_grid(c, st.L);
      g.rebuild = rb;
      grid = g;
      d.cgrid[rep] = g;
    }
  }
  __syncthreads();
  if (!grid.rebuild) return;
  const CellGrid g = grid;
  const int ncell = g.nx * g.ny * g.nz;
  if (ncell == 1) return;   // not cut: the list build scans every molecule
  const int tid = threadIdx.x, T = blockDim.x;
  for (int k = tid; k < ncell; k += T) cnt[k] = 0;
  __syncthreads();
  const int4* com = d.com + c.mol_off;
  for (int li = tid; li < c.nmol; li += T) atomicAdd(&cnt[cell_of(com[li], g)], 1);
  __syncthreads();
  // exclusive scan of the counts: a contiguous run of cells per thread
  const int per = (ncell + T - 1) / T;
  const int k0 = min(tid * per, ncell), k1 = min(k0 + per, ncell);
  int run = 0;
  for (int k = k0; k < k1; k++) run += cnt[k];
  int incl = run;
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if ((tid & 31) >= o) incl += y;
  }
  if ((tid & 31) == 31) wsum[tid >> 5] = incl;
  __syncthreads();
  int base = incl - run;
  for (int w = 0; w < (tid >> 5); w++) base += wsum[w];
  int* cs = d.cell_start + (long long)rep * (kMaxCells + 1);
  for (int k = k0; k < k1; k++) {
    const int n = cnt[k];
    cnt[k] = base;
    cs[k] = base;
    base += n;
  }
  if (tid == 0) cs[ncell] = c.nmol;
  __syncthreads();
  int4* cm = d.cell_com + c.mol_off;
  for (int li = tid; li < c.nmol; li += T) {
    int4 x = com[li];
    const int pos = atomicAdd(&cnt[cell_of(x, g)], 1);
    x.w = li;
    cm[pos] = x;
  }
}

// Neighbour-list rebuild for the molecules of this tile, one lane per molecule
// (build_lists, the FP64 form; the FP32 form's build_lists_f32 below gives the
// same lists with four lanes per molecule).  The list of molecule i holds, in
// ascending j, every j that passes the list test (below):
//  * a replica not cut into cells (CellGrid 1 x 1 x 1): every molecule of the
//    replica is tested, 128 candidates at a time from shared memory (all lanes
//    read the same candidate: a broadcast), which emits them in ascending j;
//  * a replica cut into cells (k_replica_head): molecule i tests the molecules
//    of its neighbouring cells only (their centres, sorted by cell, carry the
//    local index in .w) and sets their bits in its row of a bitmap in shared
//    memory (`win` words per row: molecules [32 w0, 32 (w0 + win)) at a time),
//    then emits the set bits in ascending j -- the same list as the scan.
// FP32 form: the skin list only has to contain every pair within rcut+skin
// (pass 1 then keeps exactly the pairs within rcut), so the test is a
// conservative one in FP32 on the top 16 bits of each fixed-point difference
// (converted with the 1.5*2^23 bit trick, on the FMA pipe), against
// rcut+skin widened by the truncation error sqrt(3) L_max 2^-16 and a relative
// 1e-5.  It may keep a few pairs just beyond rcut+skin; the lists, and
// therefore the results, of pass 1 do not change.
template <int PREC>
__device__ __forceinline__ bool list_test(const int4 me, const int4 cj, float lsc0, float lsc1, float lsc2,
                                          float rl2f, double rx, double ry, double rz, const double* wj,
                                          const double* L, double rl2) {
  if (PREC == kF32) {
    const float fx = (__int_as_float(0x4B400000 + (wrap_diff(me.x, cj.x) >> 16)) - 12582912.f) * lsc0;
    const float fy = (__int_as_float(0x4B400000 + (wrap_diff(me.y, cj.y) >> 16)) - 12582912.f) * lsc1;
    const float fz = (__int_as_float(0x4B400000 + (wrap_diff(me.z, cj.z) >> 16)) - 12582912.f) * lsc2;
    return fx * fx + fy * fy + fz * fz < rl2f;
  }
  double dx = (rx - wj[0]) * L[0];
  double dy = (ry - wj[1]) * L[1];
  double dz = (rz - wj[2]) * L[2];
  if (dx >= 0.5 * L[0]) dx -= L[0];
  if (dx < -0.5 * L[0]) dx += L[0];
  if (dy >= 0.5 * L[1]) dy -= L[1];
  if (dy < -0.5 * L[1]) dy += L[1];
  if (dz >= 0.5 * L[2]) dz -= L[2];
  if (dz < -0.5 * L[2]) dz += L[2];
  return dx * dx + dy * dy + dz * dz < rl2;
}

__device__ void build_lists(const DevPtrs& d, const RepConst& c, const Tile& t, const double* L,
                            uint16_t* nb, int tile_size, uint32_t* bm, int win) {
  __shared__ double4 cand[128];
  const int i = threadIdx.x;
  const bool valid = i < t.count;
  const int li = t.start + i;
  const double rl = c.rc + c.skin;
  const double rl2 = rl * rl;
  const int4* com = d.com + c.mol_off;   // cell coordinates of the centres
  const double* pk = reinterpret_cast<const double*>(d.pack) + c.pack_off;
  int4 me = make_int4(0, 0, 0, 0);
  double rx = 0, ry = 0, rz = 0;
  if (valid) {
    me = com[li];
    rx = pk[(long long)li * c.pack_stride];
    ry = pk[(long long)li * c.pack_stride + 1];
    rz = pk[(long long)li * c.pack_stride + 2];
  }
  const CellGrid g = d.cgrid[t.rep];
  int cnt = 0;
  if (g.nx * g.ny * g.nz == 1) {
    // every molecule, 128 at a time through shared memory (uniform over the block)
    for (int base = 0; base < c.nmol; base += 128) {
      __syncthreads();
      for (int k = threadIdx.x; k < 128 && base + k < c.nmol; k += blockDim.x) {
        const double* w = pk + (long long)(base + k) * c.pack_stride;
        cand[k] = make_double4(w[0], w[1], w[2], 0);
      }
      __syncthreads();
      if (valid) {
        const int nk = min(128, c.nmol - base);
        for (int k = 0; k < nk; k++) {
          const int j = base + k;
          const bool in = list_test<kF64>(me, make_int4(0, 0, 0, 0), 0.f, 0.f, 0.f, 0.f, rx, ry, rz,
                                          reinterpret_cast<const double*>(&cand[k]), L, rl2);
          if (j != li && in) {
            if (cnt < c.nbr_cap) nb[(long long)cnt * tile_size] = (uint16_t)j;
            cnt++;
          }
        }
      }
    }
  } else if (valid) {
    uint32_t* row = bm + i * (win | 1);   // odd row length: the lanes' words fall in distinct banks
    const int W = (c.nmol + 31) >> 5;
    const int cx = cell_coord(me.x, g.nx), cy = cell_coord(me.y, g.ny), cz = cell_coord(me.z, g.nz);
    const int ox = (g.nx == 1) ? 0 : 1, oy = (g.ny == 1) ? 0 : 1, oz = (g.nz == 1) ? 0 : 1;
    const int* cs = d.cell_start + (long long)t.rep * (kMaxCells + 1);
    const int4* cm = d.cell_com + c.mol_off;
    for (int w0 = 0; w0 < W; w0 += win) {
      const int nw = min(win, W - w0);
      for (int w = 0; w < nw; w++) row[w] = 0u;
      const int jlo = 32 * w0, jhi = 32 * (w0 + nw);
      for (int dz = -oz; dz <= oz; dz++) {
        int zc = cz + dz;
        zc += (zc < 0) ? g.nz : 0;
        zc -= (zc >= g.nz) ? g.nz : 0;
        for (int dy = -oy; dy <= oy; dy++) {
          int yc = cy + dy;
          yc += (yc < 0) ? g.ny : 0;
          yc -= (yc >= g.ny) ? g.ny : 0;
          for (int dx = -ox; dx <= ox; dx++) {
            int xc = cx + dx;
            xc += (xc < 0) ? g.nx : 0;
            xc -= (xc >= g.nx) ? g.nx : 0;
            const int cell = (zc * g.ny + yc) * g.nx + xc;
            const int e = cs[cell + 1];
            for (int k = cs[cell]; k < e; k++) {
              const int4 cj = cm[k];
              const int j = cj.w;
              if (j < jlo || j >= jhi || j == li) continue;
              if (list_test<kF64>(me, cj, 0.f, 0.f, 0.f, 0.f, rx, ry, rz, pk + (long long)j * c.pack_stride, L,
                                  rl2))
                row[(j - jlo) >> 5] |= 1u << (j & 31);
            }
          }
        }
      }
      for (int w = 0; w < nw; w++) {
        uint32_t bits = row[w];
        while (bits) {
          const int j = jlo + 32 * w + (__ffs(bits) - 1);
          bits &= bits - 1u;
          if (cnt < c.nbr_cap) nb[(long long)cnt * tile_size] = (uint16_t)j;
          cnt++;
        }
      }
    }
  }
  if (valid) {
    if (cnt > c.nbr_cap) {
      atomicOr(d.err, kErrNbrOverflow);
      atomicMax(&d.status[t.rep], 8);
      cnt = c.nbr_cap;
    }
    d.nbr_cnt[c.mol_off + li] = cnt;
  }
}

// FP32 skin-list build for the list kernel, kListLanes lanes per molecule
// (molecule slot threadIdx.x / kListLanes, lane sub = threadIdx.x % kListLanes).
// The lists are entry for entry those that build_lists gives with one lane per
// molecule (the FP64 form still builds its lists that way):
//  * all-molecule scan: lane sub tests candidates sub, sub + 4, ... of each
//    128-molecule chunk staged in shared memory, and a ballot places the kept
//    ones in ascending j;
//  * cell lists: the lanes split each neighbouring cell's molecules and set
//    the molecule's bitmap row with shared-memory atomics; the row is then
//    emitted in ascending j, lane sub taking words sub, sub + 4, ..., placed by
//    a prefix of their popcounts over the group.
// Returns the list length (equal on the group's lanes); lane 0 stores it.
__device__ int build_lists_f32(const DevPtrs& d, const RepConst& c, const Tile& t, const double* L,
                               uint16_t* nb, int T, uint32_t* bm, int win) {
  __shared__ int4 cand[128];
  const int i = threadIdx.x / kListLanes, sub = threadIdx.x % kListLanes, lane = threadIdx.x & 31;
  const unsigned below = (1u << sub) - 1u;
  const bool valid = i < t.count;
  const int li = t.start + i;
  const float lsc0 = (float)(L[0] * (1.0 / 65536.0)), lsc1 = (float)(L[1] * (1.0 / 65536.0)),
              lsc2 = (float)(L[2] * (1.0 / 65536.0));
  const double rw = list_test_radius(c, L);
  const float rl2f = (float)(rw * rw);
  const int4* com = d.com + c.mol_off;
  const int4 me = valid ? com[li] : make_int4(0, 0, 0, 0);
  const CellGrid g = d.cgrid[t.rep];
  int cnt = 0;
  if (g.nx * g.ny * g.nz == 1) {
    for (int base = 0; base < c.nmol; base += 128) {   // uniform over the block
      __syncthreads();
      for (int k = threadIdx.x; k < 128 && base + k < c.nmol; k += blockDim.x) cand[k] = com[base + k];
      __syncthreads();
      const int nk = min(128, c.nmol - base);
      for (int k0 = 0; k0 < nk; k0 += kListLanes) {
        const int k = k0 + sub, j = base + k;
        const bool in = valid && k < nk && j != li &&
                        list_test<kF32>(me, cand[k], lsc0, lsc1, lsc2, rl2f, 0.0, 0.0, 0.0, nullptr, L, 0.0);
        const unsigned gb = group_bits(__ballot_sync(0xffffffffu, in), lane);
        if (in) {
          const int pos = cnt + __popc(gb & below);
          if (pos < c.nbr_cap) nb[(long long)pos * T] = (uint16_t)j;
        }
        cnt += __popc(gb);
      }
    }
  } else {
    uint32_t* row = bm + i * (win | 1);   // odd row length: the molecules' words fall in distinct banks
    const int W = (c.nmol + 31) >> 5;
    const int cx = cell_coord(me.x, g.nx), cy = cell_coord(me.y, g.ny), cz = cell_coord(me.z, g.nz);
    const int ox = (g.nx == 1) ? 0 : 1, oy = (g.ny == 1) ? 0 : 1, oz = (g.nz == 1) ? 0 : 1;
    const int* cs = d.cell_start + (long long)t.rep * (kMaxCells + 1);
    const int4* cm = d.cell_com + c.mol_off;
    for (int w0 = 0; w0 < W; w0 += win) {   // uniform over the block
      const int nw = min(win, W - w0);
      for (int w = sub; w < nw; w += kListLanes) row[w] = 0u;
      __syncwarp();
      const int jlo = 32 * w0, jhi = 32 * (w0 + nw);
      if (valid) {
        for (int dz = -oz; dz <= oz; dz++) {
          int zc = cz + dz;
          zc += (zc < 0) ? g.nz : 0;
          zc -= (zc >= g.nz) ? g.nz : 0;
          for (int dy = -oy; dy <= oy; dy++) {
            int yc = cy + dy;
            yc += (yc < 0) ? g.ny : 0;
            yc -= (yc >= g.ny) ? g.ny : 0;
            for (int dx = -ox; dx <= ox; dx++) {
              int xc = cx + dx;
              xc += (xc < 0) ? g.nx : 0;
              xc -= (xc >= g.nx) ? g.nx : 0;
              const int cell = (zc * g.ny + yc) * g.nx + xc;
              const int e = cs[cell + 1];
              for (int k = cs[cell] + sub; k < e; k += kListLanes) {
                const int4 cj = cm[k];
                const int j = cj.w;
                if (j < jlo || j >= jhi || j == li) continue;
                if (list_test<kF32>(me, cj, lsc0, lsc1, lsc2, rl2f, 0.0, 0.0, 0.0, nullptr, L, 0.0))
                  atomicOr(&row[(j - jlo) >> 5], 1u << (j & 31));
              }
            }
          }
        }
      }
      __syncwarp();
      for (int w = 0; w < nw; w += kListLanes) {   // uniform over the block
        const uint32_t word = (w + sub < nw) ? row[w + sub] : 0u;
        const int n = __popc(word);
        int incl = n;   // inclusive prefix of n over the group's lanes
#pragma unroll
        for (int o = 1; o < kListLanes; o <<= 1) {
          const int y = __shfl_up_sync(0xffffffffu, incl, o, kListLanes);
          if (sub >= o) incl += y;
        }
        int pos = cnt + incl - n;
        uint32_t bits = word;
        while (bits) {
          const int j = jlo + 32 * (w + sub) + (__ffs(bits) - 1);
          bits &= bits - 1u;
          if (pos < c.nbr_cap) nb[(long long)pos * T] = (uint16_t)j;
          pos++;
        }
        cnt += __shfl_sync(0xffffffffu, incl, kListLanes - 1, kListLanes);
      }
      __syncwarp();   // the row is cleared again for the next window
    }
  }
  if (cnt > c.nbr_cap) {
    if (valid && sub == 0) {
      atomicOr(d.err, kErrNbrOverflow);
      atomicMax(&d.status[t.rep], 8);
    }
    cnt = c.nbr_cap;
  }
  if (valid && sub == 0) d.nbr_cnt[c.mol_off + li] = cnt;
  return cnt;
}

// Accumulators of one molecule i.
struct IAcc {
  double fs[kMaxSites][3];   // site forces (switched pair terms + wall on site 0)
  double fc[3];              // switching correction -E dS/dr r^ (acts on the molecule only)
  double vir[3], lj, clmb;
  long long npair;
};

// FP32 pair loop over i's neighbour list, in two passes run by two kernels.
// Pass 1 (k_force_lists) scans the (rcut + skin) list and writes the neighbours
// within rcut, in the list's ascending-j order, to i's column of the per-step
// list `nbt` (same layout and capacity as the skin list; it cannot overflow).  Under the
// per-site minimum image (SIMG, below) it splits them: pairs whose COM vector
// keeps every site-pair component clear of +-L/2 ("far", from the front of the
// column) need no per-site image at all; the others ("near", from the back)
// get the per-site image.  Pass 2 computes exactly those pairs, so the lanes of
// a warp stay converged (no cutoff branch) and differ only in their counts
// (k_force_pairs).  Pass 1 runs in its own light kernel, whose occupancy hides
// the latency of its gathered loads; pass 2 is register-heavy.
// Pair math in FP32 (rsqrt on the SFU plus one Newton step); partial sums in
// FP32 over 32 pairs, then FP64 accumulation into this thread's slots of `acc`
// (shared memory, field f at acc[f * blockDim.x + threadIdx.x]: 3S site-force
// components, 3 switching-correction, 3 virial, LJ, Coulomb).  The pairs within
// rcut, their far/near class and order, and their grouping by 32 depend only
// on the positions, not on when the skin list was built.  The next
// neighbour's index is read one pair ahead of its use.
// SIMG: apply the minimum image to every site pair as the reference does
// (src/force_calculator.cxx:737-741).  It changes the result only when a box
// length is below 2 (rc + 2 site_reach); the caller enables it just then.
struct F32Const {
  float qq[kMaxSites][kMaxSites];
  float Ls[3], Lf[3], hL[3];
  double L[3];
};

// Per-site minimum image (SIMG) flips a site-pair vector by a box length where
// one of its components crosses +-L/2, so the FP32 and FP64 forms must take the
// same image there.  A site pair with a component within kImageTol of L/2
// (FP32 rounding of the site vector is below ~4e-6 A) is left out of the pair
// loop (its vector is set far away, so its terms vanish) and added afterwards
// by site_pair_exact: the image is decided with the FP64 form's arithmetic
// (pair_loop_f64: COM vector from the FP64 box fractions, site offsets R(q) b
// in FP64), then the terms are evaluated as in the loop.  Up to kMaxDefer such
// site pairs per molecule and step are deferred; further ones (never seen in
// practice) keep the FP32 image.
constexpr float kImageTol = 2e-5f;
constexpr int kMaxDefer = 2;

template <int S, int C0>
__device__ __noinline__ void site_pair_exact(const DevPtrs& d, const RepConst& c, const F32Const& k32, int li,
                                             int code, double* acc) {
  const int j = code >> 8, kk = (code >> 4) & 15, l = code & 15;
  const int T = blockDim.x, tid = threadIdx.x;
  const int N = d.N, gi = c.mol_off + li, gj = c.mol_off + j;
  const double* L = k32.L;
  // COM vector and switch exactly as the FP32 loop forms them
  const uint32_t* base = reinterpret_cast<const uint32_t*>(d.pack) + c.pack_off;
  const int stride = c.pack_stride;
  const int* wi = reinterpret_cast<const int*>(base + (long long)li * stride);
  const int* wj = reinterpret_cast<const int*>(base + (long long)j * stride);
  const float dx = (float)wrap_diff(wi[0], wj[0]) * k32.Ls[0];
  const float dy = (float)wrap_diff(wi[1], wj[1]) * k32.Ls[1];
  const float dz = (float)wrap_diff(wi[2], wj[2]) * k32.Ls[2];
  const float r2 = dx * dx + dy * dy + dz * dz;
  const float rinv = rsqrtf(r2);
  const float r = r2 * rinv;
  const float rc = (float)c.rc, rs = (float)c.rs, coef = (float)c.coef_sw;
  float sw = 1.f, dsw = 0.f;
  if (r > rs) {
    const float r01c = r - rc, r01l = r - rs;
    sw = coef * r01c * r01c * r01c * (10.f * r01l * r01l - 5.f * r01l * r01c + r01c * r01c);
    dsw = coef * 30.f * r01c * r01c * r01l * r01l;
  }
  // the site vector with the FP64 form's image
  double qi[4], qj[4], si[3], sj[3];
  for (int x = 0; x < 4; x++) { qi[x] = d.q[x * N + gi]; qj[x] = d.q[x * N + gj]; }
  body_to_space(qi, c.body[kk], si);
  body_to_space(qj, c.body[l], sj);
  float v[3];
  for (int x = 0; x < 3; x++) {
    double gr = (d.r[x * N + gi] - d.r[x * N + gj]) * L[x];
    if (gr >= 0.5 * L[x]) gr -= L[x];
    if (gr < -0.5 * L[x]) gr += L[x];
    double rv = gr + si[x] - sj[x];
    if (rv >= 0.5 * L[x]) rv -= L[x];
    if (rv < -0.5 * L[x]) rv += L[x];
    v[x] = (float)rv;
  }
  const float rr = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
  float ri = rsqrtf(rr);
  ri = ri * fmaf(-0.5f * rr * ri, ri, 1.5f);
  const float ri2 = ri * ri;
  float ftmp = 0.f, elj = 0.f, ecl = 0.f;
  if (kk == 0 && l == 0) {
    float s6 = (float)c.sgm2 * ri2;
    s6 = s6 * s6 * s6;
    elj = (float)(4.0 * c.eps) * s6 * (s6 - 1.f);
    ftmp += (float)(48.0 * c.eps) * s6 * (s6 - 0.5f) * ri2;
  }
  if (kk >= C0 && l >= C0) {
    ecl = k32.qq[kk][l] * ri;
    ftmp += ecl * ri2;
  }
  ftmp *= sw;
  const float t[3] = {v[0] * ftmp, v[1] * ftmp, v[2] * ftmp};
  const float g = dsw * rinv * (elj + ecl);
  const float cv[3] = {-dx * g, -dy * g, -dz * g};
  const float dv[3] = {dx, dy, dz};
  for (int x = 0; x < 3; x++) {
    acc[(3 * kk + x) * T + tid] += (double)t[x];
    acc[(3 * S + x) * T + tid] += (double)cv[x];
    acc[(3 * S + 3 + x) * T + tid] += (double)((t[x] + cv[x]) * dv[x]);
  }
  acc[(3 * S + 6) * T + tid] += (double)(sw * elj);
  acc[(3 * S + 7) * T + tid] += (double)(sw * ecl);
}

// Pass 1 for molecule li of tile t, run by its kListLanes lanes (sub = 0..3):
// the neighbours of its (rcut + skin) list that are within rcut, in ascending
// j, into its column of `nt` -- far pairs from the front, near pairs (SIMG
// only) from the back.  Lane sub tests list entries sub, sub + 4, ...; a round
// of the group covers four consecutive entries, and the kept ones are placed by
// a ballot in list order, so the lists equal those of one lane walking the
// list in turn.  Four rounds per batch, so that their record loads are in
// flight together.  Lane 0 stores nfar | nnear << 16 in d.nt_cnt.  Every lane
// of the warp runs the warp's longest list (ballots need the whole warp).
template <bool SIMG>
__device__ void tight_lists_f32(const DevPtrs& d, const RepConst& c, int li, bool valid, int sub,
                                const double* L, const uint16_t* nb, uint16_t* nt, int cnt, int T) {
  const int4* base = d.com + c.mol_off;   // compact centres: 16 B per molecule, L1-resident
  const float Ls0 = (float)(L[0] * kFixInv), Ls1 = (float)(L[1] * kFixInv), Ls2 = (float)(L[2] * kFixInv);
  const float rc2 = (float)(c.rc * c.rc);
  const int4 ui = valid ? __ldg(base + li) : make_int4(0, 0, 0, 0);
  const int xi = ui.x, yi = ui.y, zi = ui.z;
  // far bound: |d_x| below it keeps every site-pair component below L/2 - kImageTol
  float bnd0 = 0.f, bnd1 = 0.f, bnd2 = 0.f;
  if (SIMG) {
    const float m = 2.f * (float)c.site_reach + kImageTol + 1e-3f;
    bnd0 = 0.5f * (float)L[0] - m; bnd1 = 0.5f * (float)L[1] - m; bnd2 = 0.5f * (float)L[2] - m;
  }
  const int lane = threadIdx.x & 31;
  const unsigned below = (1u << sub) - 1u;
  const int back = c.nbr_cap - 1;
  int nfar = 0, nnear = 0;
  const int rounds = __reduce_max_sync(0xffffffffu, (cnt + kListLanes - 1) / kListLanes);
  constexpr int B = 4;
  for (int r0 = 0; r0 < rounds; r0 += B) {
    int j[B];
    int4 u[B];
#pragma unroll
    for (int m = 0; m < B; m++) {
      const int k = (r0 + m) * kListLanes + sub;
      j[m] = (k < cnt) ? (int)nb[(long long)k * T] : -1;
    }
#pragma unroll
    for (int m = 0; m < B; m++) u[m] = (j[m] >= 0) ? __ldg(base + j[m]) : ui;
#pragma unroll
    for (int m = 0; m < B; m++) {
      const float dx = (float)wrap_diff(xi, u[m].x) * Ls0, dy = (float)wrap_diff(yi, u[m].y) * Ls1,
                  dz = (float)wrap_diff(zi, u[m].z) * Ls2;
      const bool in = j[m] >= 0 && dx * dx + dy * dy + dz * dz <= rc2;
      const bool near = SIMG && in && (fabsf(dx) >= bnd0 || fabsf(dy) >= bnd1 || fabsf(dz) >= bnd2);
      const unsigned gf = group_bits(__ballot_sync(0xffffffffu, in && !near), lane);
      if (in && !near) nt[(long long)(nfar + __popc(gf & below)) * T] = (uint16_t)j[m];
      nfar += __popc(gf);
      if (SIMG) {
        const unsigned gn = group_bits(__ballot_sync(0xffffffffu, near), lane);
        if (near) nt[(long long)(back - nnear - __popc(gn & below)) * T] = (uint16_t)j[m];
        nnear += __popc(gn);
      }
    }
  }
  if (valid && sub == 0) d.nt_cnt[c.mol_off + li] = nfar | (nnear << 16);
}

template <int S, int C0, bool SIMG>
__device__ void pair_loop_f32(const DevPtrs& d, const RepConst& c, const F32Const& k32, int li,
                              const uint16_t* nt, int lstride, int nfar, int nnear, int p0, int p1,
                              double* acc) {
  constexpr int STRIDE = ((3 + 3 * S) + 3) / 4 * 4;
  constexpr int NV = STRIDE / 4;
  const int T = blockDim.x, tid = threadIdx.x;   // accumulator slots
  const uint4* base = reinterpret_cast<const uint4*>(reinterpret_cast<const uint32_t*>(d.pack) + c.pack_off);
  const float Ls0 = k32.Ls[0], Ls1 = k32.Ls[1], Ls2 = k32.Ls[2];
  int xi, yi, zi;
  float si[S][3];
  {
    uint32_t wi[STRIDE];
#pragma unroll
    for (int k = 0; k < NV; k++) {
      const uint4 u = __ldg(base + (long long)li * NV + k);
      wi[4 * k] = u.x; wi[4 * k + 1] = u.y; wi[4 * k + 2] = u.z; wi[4 * k + 3] = u.w;
    }
    xi = (int)wi[0]; yi = (int)wi[1]; zi = (int)wi[2];
#pragma unroll
    for (int k = 0; k < S; k++)
#pragma unroll
      for (int x = 0; x < 3; x++) si[k][x] = __uint_as_float(wi[3 + 3 * k + x]);
  }
  const int back = c.nbr_cap - 1;
  const float rc = (float)c.rc, rs = (float)c.rs;
  const float coef = (float)c.coef_sw;
  const float sgm2 = (float)c.sgm2, eps4 = (float)(4.0 * c.eps), eps48 = (float)(48.0 * c.eps);

  float fs[S][3], fc[3], fv[3], flj, fcl;
  auto zero = [&]() {
#pragma unroll
    for (int k = 0; k < S; k++) fs[k][0] = fs[k][1] = fs[k][2] = 0.f;
    fc[0] = fc[1] = fc[2] = 0.f;
    fv[0] = fv[1] = fv[2] = 0.f;
    flj = fcl = 0.f;
  };
  auto flush = [&]() {
#pragma unroll
    for (int k = 0; k < S; k++)
#pragma unroll
      for (int x = 0; x < 3; x++) acc[(3 * k + x) * T + tid] += (double)fs[k][x];
#pragma unroll
    for (int x = 0; x < 3; x++) {
      acc[(3 * S + x) * T + tid] += (double)fc[x];
      acc[(3 * S + 3 + x) * T + tid] += (double)fv[x];
    }
    acc[(3 * S + 6) * T + tid] += (double)flj;
    acc[(3 * S + 7) * T + tid] += (double)fcl;
  };
  zero();
  int done = 0;                       // pairs accumulated (partial sums close every 32)
  int ndef = 0, def0 = 0, def1 = 0;   // deferred site pairs (near pass only)

  // pass 2: `n` pairs of the list starting at column slot `pos0`, stepping `dir`;
  // IMG: per-site minimum image with exact ties (near pairs)
  auto run = [&](auto img, int n, int pos0, int dir) {
    constexpr bool IMG = decltype(img)::value;
    const float hL0 = k32.hL[0], hL1 = k32.hL[1], hL2 = k32.hL[2];
    const float Lf0 = k32.Lf[0], Lf1 = k32.Lf[1], Lf2 = k32.Lf[2];
    // the next neighbour's index one pair ahead; the record at the top of the
    // iteration (a record held in registers one pair ahead was 5 % slower)
    int jnext = (n > 0) ? nt[(long long)pos0 * lstride] : 0;
    for (int k = 0; k < n; k++) {
      const int jcur = jnext;
      if (k + 1 < n) jnext = nt[(long long)(pos0 + dir * (k + 1)) * lstride];
      uint32_t wj[STRIDE];
#pragma unroll
      for (int m = 0; m < NV; m++) {
        const uint4 u = __ldg(base + (long long)jcur * NV + m);
        wj[4 * m] = u.x; wj[4 * m + 1] = u.y; wj[4 * m + 2] = u.z; wj[4 * m + 3] = u.w;
      }
      const float dx = (float)wrap_diff(xi, (int)wj[0]) * Ls0;
      const float dy = (float)wrap_diff(yi, (int)wj[1]) * Ls1;
      const float dz = (float)wrap_diff(zi, (int)wj[2]) * Ls2;
      const float r2 = dx * dx + dy * dy + dz * dz;
      const float rinv = rsqrtf(r2);
      const float r = r2 * rinv;
      float sw = 1.f, dsw = 0.f;
      if (r > rs) {
        const float r01c = r - rc, r01l = r - rs;
        sw = coef * r01c * r01c * r01c * (10.f * r01l * r01l - 5.f * r01l * r01c + r01c * r01c);
        dsw = coef * 30.f * r01c * r01c * r01l * r01l;
      }
      float elj = 0.f, ecl = 0.f;
      float fpx = 0.f, fpy = 0.f, fpz = 0.f;
#pragma unroll
      for (int kk = 0; kk < S; kk++) {
        if (kk != 0 && kk < C0) continue;
        const float ax = dx + si[kk][0], ay = dy + si[kk][1], az = dz + si[kk][2];
        float tx = 0.f, ty = 0.f, tz = 0.f;
#pragma unroll
        for (int l = 0; l < S; l++) {
          const bool lj_pair = (kk == 0 && l == 0);
          const bool cl_pair = (kk >= C0 && l >= C0);
          if (!lj_pair && !cl_pair) continue;
          float x = ax - __uint_as_float(wj[3 + 3 * l]);
          float y = ay - __uint_as_float(wj[3 + 3 * l + 1]);
          float z = az - __uint_as_float(wj[3 + 3 * l + 2]);
          if (IMG) {
            if ((fabsf(fabsf(x) - hL0) < kImageTol || fabsf(fabsf(y) - hL1) < kImageTol ||
                 fabsf(fabsf(z) - hL2) < kImageTol) && ndef < kMaxDefer) {
              const int code = (jcur << 8) | (kk << 4) | l;
              if (ndef == 0) def0 = code; else def1 = code;
              ndef++;
              x = y = z = 1e18f;   // this site pair's terms vanish here; added exactly below
            }
            if (x >= hL0) x -= Lf0;
            if (x < -hL0) x += Lf0;
            if (y >= hL1) y -= Lf1;
            if (y < -hL1) y += Lf1;
            if (z >= hL2) z -= Lf2;
            if (z < -hL2) z += Lf2;
          }
          const float rr = x * x + y * y + z * z;
          float ri = rsqrtf(rr);
          ri = ri * fmaf(-0.5f * rr * ri, ri, 1.5f);   // one Newton step: ~0.5 ulp
          const float ri2 = ri * ri;
          float ftmp = 0.f;
          if (lj_pair) {
            float s6 = sgm2 * ri2;
            s6 = s6 * s6 * s6;
            elj += eps4 * s6 * (s6 - 1.f);
            ftmp += eps48 * s6 * (s6 - 0.5f) * ri2;
          }
          if (cl_pair) {
            const float e = k32.qq[kk][l] * ri;
            ecl += e;
            ftmp += e * ri2;
          }
          tx += x * ftmp; ty += y * ftmp; tz += z * ftmp;
        }
        // the switch multiplies the site forces once per site (FFMA into the sums)
        fs[kk][0] = fmaf(sw, tx, fs[kk][0]);
        fs[kk][1] = fmaf(sw, ty, fs[kk][1]);
        fs[kk][2] = fmaf(sw, tz, fs[kk][2]);
        fpx += tx; fpy += ty; fpz += tz;
      }
      const float e = elj + ecl;
      const float g = dsw * rinv * e;
      const float cx = -dx * g, cy = -dy * g, cz = -dz * g;
      fc[0] += cx; fc[1] += cy; fc[2] += cz;
      fv[0] += fmaf(fpx, sw, cx) * dx;
      fv[1] += fmaf(fpy, sw, cy) * dy;
      fv[2] += fmaf(fpz, sw, cz) * dz;
      flj += sw * elj;
      fcl += sw * ecl;
      if ((++done & 31) == 0) { flush(); zero(); }
    }
  };
  // positions [p0, p1) of the sequence far pairs (rows 0..) then near pairs (rows back, back-1, ..)
  const int f1 = min(p1, nfar);
  run(std::false_type{}, max(f1 - p0, 0), p0, 1);
  if (SIMG) {
    const int q0 = max(p0, nfar);
    run(std::true_type{}, max(p1 - q0, 0), back - (q0 - nfar), -1);
  }
  flush();
  if (SIMG && ndef > 0) {
    site_pair_exact<S, C0>(d, c, k32, li, def0, acc);
    if (ndef > 1) site_pair_exact<S, C0>(d, c, k32, li, def1, acc);
  }
}

template <int S, int C0, bool SIMG>
__device__ void pair_loop_f64(const DevPtrs& d, const RepConst& c, const Tile& t, const double* L,
                              const uint16_t* nb, int cnt, IAcc& a) {
  constexpr int STRIDE = ((3 + 3 * S) + 1) / 2 * 2;
  const int li = t.start + threadIdx.x;
  const double* base = reinterpret_cast<const double*>(d.pack) + c.pack_off;
  double wi[STRIDE];
#pragma unroll
  for (int k = 0; k < STRIDE; k++) wi[k] = base[(long long)li * STRIDE + k];
  const double rc = c.rc, rl = c.rs, coef = c.coef_sw, rc2 = c.rc * c.rc;
  for (int k = 0; k < cnt; k++) {
    const int j = nb[(long long)k * blockDim.x];
    const double* wj = base + (long long)j * STRIDE;
    double gr[3];
    for (int x = 0; x < 3; x++) {
      gr[x] = (wi[x] - wj[x]) * L[x];
      if (gr[x] >= 0.5 * L[x]) gr[x] -= L[x];
      if (gr[x] < -0.5 * L[x]) gr[x] += L[x];
    }
    const double r02 = gr[0] * gr[0] + gr[1] * gr[1] + gr[2] * gr[2];
    if (r02 > rc2) continue;
    a.npair++;
    const double r01 = sqrt(r02);
    double sw = 1.0, dsw = 0.0;
    if (r01 > rl) {
      const double r01c = r01 - rc, r01l = r01 - rl;
      sw = coef * r01c * r01c * r01c * (10.0 * r01l * r01l - 5.0 * r01l * r01c + r01c * r01c);
      dsw = coef * 30.0 * r01c * r01c * r01l * r01l;
    }
    double dswr[3];
    for (int x = 0; x < 3; x++) dswr[x] = gr[x] * (dsw / r01);
#pragma unroll
    for (int kk = 0; kk < S; kk++) {
      if (kk != 0 && kk < C0) continue;
      double e = 0.0, f[3] = {0.0, 0.0, 0.0};
#pragma unroll
      for (int l = 0; l < S; l++) {
        const bool lj_pair = (kk == 0 && l == 0);
        const bool cl_pair = (kk >= C0 && l >= C0);
        if (!lj_pair && !cl_pair) continue;
        double rv[3];
        for (int x = 0; x < 3; x++) {
          rv[x] = gr[x] + wi[3 + 3 * kk + x] - wj[3 + 3 * l + x];
          if (SIMG) {
            if (rv[x] >= 0.5 * L[x]) rv[x] -= L[x];
            if (rv[x] < -0.5 * L[x]) rv[x] += L[x];
          }
        }
        const double rr = rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2];
        const double r02i = 1.0 / rr;
        const double r01i = sqrt(r02i);
        const double qq = cl_pair ? c.qq[kk][l] : 0.0;
        double elj = 0.0, flj = 0.0;
        if (lj_pair) {
          double rs06i = c.sgm2 * r02i;
          rs06i = rs06i * rs06i * rs06i;
          elj = 4.0 * c.eps * rs06i * (rs06i - 1.0);
          flj = 48.0 * c.eps * rs06i * (rs06i - 0.5) * r02i;
        }
        const double ecl = qq * r01i;
        a.lj += sw * elj;
        a.clmb += sw * ecl;
        const double ftmp = (flj + qq * r01i * r02i) * sw;
        e += elj + ecl;
        for (int x = 0; x < 3; x++) {
          f[x] += rv[x] * ftmp;
          a.fs[kk][x] += rv[x] * ftmp;
        }
      }
      for (int x = 0; x < 3; x++) {
        const double cx = -dswr[x] * e;
        a.fc[x] += cx;
        a.vir[x] += (f[x] + cx) * gr[x];
      }
    }
  }
}

// Wall on the oxygen site and A2M for molecule g (FP64): writes d.f, d.n.
template <int S>
__device__ void finish_molecule(const DevPtrs& d, const RepConst& c, int g, const double* L, IAcc& a,
                                double& wall_e) {
  const int N = d.N;
  double q[4], r[3];
  for (int x = 0; x < 4; x++) q[x] = d.q[x * N + g];
  for (int x = 0; x < 3; x++) r[x] = d.r[x * N + g];
  // wall on the oxygen site (ForceCalculator::Confined, src/force_calculator.cxx:1527-1566;
  // slit: src/remdgpu.cu:1708-1720)
  if (c.confined > 0) {
    double o[3];
    body_to_space(q, c.body[0], o);
    const double2* fw = reinterpret_cast<const double2*>(d.wall) + c.wall_off;
    const double dr = c.wall_dr;
    if (c.confined == 1) {
      const double x = r[0] * L[0] + o[0] - L[0] * 0.5;
      const double y = r[1] * L[1] + o[1] - L[1] * 0.5;
      const double r01 = sqrt(x * x + y * y);
      int idx = (r01 >= 0.0) ? (int)fmin(r01 / dr, (double)(c.nfwall - 2)) : 0;   // NaN -> 0
      const double2 w0 = fw[idx], w1 = fw[idx + 1];
      const double f = (w1.x - w0.x) / dr * (r01 - dr * idx) + w0.x;
      const double e = (w1.y - w0.y) / dr * (r01 - dr * idx) + w0.y;
      a.fs[0][0] += f * x;
      a.fs[0][1] += f * y;
      wall_e = e;
    } else {
      const double z = r[2] * L[2] + o[2] - 0.5 * L[2];
      const double za = fabs(z);
      const double dir = (za != 0.0) ? z / za : 1.0;
      int idx = (za >= 0.0) ? (int)fmin(za / dr, (double)(c.nfwall - 2)) : 0;     // NaN -> 0
      const double2 w0 = fw[idx], w1 = fw[idx + 1];
      const double f = (w1.x - w0.x) / dr * (za - dr * idx) + w0.x;
      const double e = (w1.y - w0.y) / dr * (za - dr * idx) + w0.y;
      a.fs[0][2] += f * dir;
      wall_e = e;
    }
  }
  // A2M: molecular force and body torque (src/molecules.cxx:447-475)
  double F[3] = {a.fc[0], a.fc[1], a.fc[2]};
  double nq[4] = {0, 0, 0, 0};
#pragma unroll
  for (int k = 0; k < S; k++) {
    for (int x = 0; x < 3; x++) F[x] += a.fs[k][x];
    double fb[3];
    space_to_body(q, a.fs[k], fb);
    const double* b = c.body[k];
    nq[0] += b[0] * fb[0] + b[1] * fb[1] + b[2] * fb[2];
    nq[1] += b[1] * fb[2] - b[2] * fb[1];
    nq[2] += b[2] * fb[0] - b[0] * fb[2];
    nq[3] += b[0] * fb[1] - b[1] * fb[0];
  }
  for (int x = 0; x < 3; x++) d.f[x * N + g] = F[x];
  for (int x = 0; x < 4; x++) d.n[x * N + g] = nq[x];
}

// Force partials of the tile's 32-molecule units (one fixed shuffle tree per warp).
__device__ inline void write_part2(const DevPtrs& d, const RepConst& c, const Tile& t, const IAcc& a,
                                   double wall_e) {
  double s6[7] = {a.lj, a.clmb, wall_e, a.vir[0], a.vir[1], a.vir[2], (double)a.npair};
  warp_sum<7>(s6);
  const int w = (t.start + threadIdx.x) >> 5;   // 32-molecule unit of the replica
  if ((threadIdx.x & 31) == 0 && w < c.nwarp) {
    Part2 p;
    p.lj = s6[0]; p.clmb = s6[1]; p.wall = s6[2];
    p.vir[0] = s6[3]; p.vir[1] = s6[4]; p.vir[2] = s6[5];
    p.npairs = (long long)llrint(s6[6]);
    p.pad = 0.0;
    d.part2[c.warp_off + w] = p;
  }
}

__device__ inline void zero_acc(IAcc& a) {
#pragma unroll
  for (int k = 0; k < kMaxSites; k++) a.fs[k][0] = a.fs[k][1] = a.fs[k][2] = 0.0;
  a.fc[0] = a.fc[1] = a.fc[2] = 0.0;
  a.vir[0] = a.vir[1] = a.vir[2] = 0.0;
  a.lj = a.clmb = 0.0;
  a.npair = 0;
}

// FP64 form: skin-list rebuild of tile t when due, with the build's reference
// centres and box.
__device__ void rebuild_tile(const DevPtrs& d, const RepConst& c, const Tile& t, int tix, const double* L,
                             uint16_t* nb, int tile_size, uint32_t* bm, int win) {
  const int i = threadIdx.x;
  const int li = t.start + i;
  build_lists(d, c, t, L, nb, tile_size, bm, win);
  if (i < t.count) {
    const double* wd = reinterpret_cast<const double*>(d.pack) + c.pack_off + (long long)li * c.pack_stride;
    d.ref_com[c.mol_off + li] = make_int4(fix_coord(wd[0]), fix_coord(wd[1]), fix_coord(wd[2]), 0);
  }
  if (i == 0)
    for (int x = 0; x < 3; x++) d.Lbuild[3 * tix + x] = L[x];
}

__device__ inline bool site_image_needed(const RepConst& c, const double* L) {
  const double reach = c.rc + 2.0 * c.site_reach;
  return (L[0] < 2.0 * reach) || (L[1] < 2.0 * reach) || (L[2] < 2.0 * reach);
}

// FP64 form: rebuild when due, pair loop, wall, A2M.
template <int S, int C0>
__device__ void force_tile_f64(const DevPtrs& d, const RepConst& c, const Tile& t, int tix, const double* L,
                               bool rebuild, int tile_size, uint32_t* bm, int win) {
  const int i = threadIdx.x;
  const int li = t.start + i;
  const int g = c.mol_off + li;
  uint16_t* nb = d.nbr + c.nbr_off + (long long)(tix - c.tile_off) * c.nbr_cap * tile_size + i;
  if (rebuild) rebuild_tile(d, c, t, tix, L, nb, tile_size, bm, win);
  IAcc a;
  zero_acc(a);
  double wall_e = 0.0;
  if (i < t.count) {
    const int cnt = d.nbr_cnt[g];
    if (site_image_needed(c, L)) pair_loop_f64<S, C0, true>(d, c, t, L, nb, cnt, a);
    else pair_loop_f64<S, C0, false>(d, c, t, L, nb, cnt, a);
    finish_molecule<S>(d, c, g, L, a, wall_e);
  }
  write_part2(d, c, t, a, wall_e);
}

// FP32 form, pass 2 + wall + A2M (the per-step list comes from k_force_lists).
// Two threads per molecule: thread (i, ch) computes positions [ch n/2, (ch+1) n/2)
// of i's n pairs, so a launch has twice the work units (a shorter tail); the
// two FP64 partials are added in chunk order.  The split is by list position
// and the list holds exactly the pairs within rcut in ascending j, so results
// depend neither on the tile size nor on the list history.
constexpr int kPairChunks = 2;

template <int S, int C0>
__device__ void force_tile_f32(const DevPtrs& d, const RepConst& c, const Tile& t, int tix, const double* L,
                               int tile_size) {
  __shared__ F32Const k32;
  extern __shared__ double acc[];   // (3S + 8) x blockDim.x FP64 accumulators
  const int B = blockDim.x;
  const int i = threadIdx.x % tile_size, ch = threadIdx.x / tile_size;
  const int li = t.start + i;
  const int g = c.mol_off + li;
  if (threadIdx.x == 0) {
    for (int k = 0; k < kMaxSites; k++)
      for (int l = 0; l < kMaxSites; l++) k32.qq[k][l] = (float)c.qq[k][l];
    for (int x = 0; x < 3; x++) {
      k32.Ls[x] = (float)(L[x] * kFixInv);
      k32.Lf[x] = (float)L[x];
      k32.hL[x] = 0.5f * (float)L[x];
      k32.L[x] = L[x];
    }
  }
  for (int f = 0; f < 3 * S + 8; f++) acc[f * B + threadIdx.x] = 0.0;
  __syncthreads();
  int npairs = 0;
  if (i < t.count) {
    const uint16_t* nt = d.nbt + c.nbr_off + (long long)(tix - c.tile_off) * c.nbr_cap * tile_size + i;
    const int nc = d.nt_cnt[g];
    const int nfar = nc & 0xffff, nnear = nc >> 16;
    npairs = nfar + nnear;
    const int p0 = (npairs * ch) / kPairChunks, p1 = (npairs * (ch + 1)) / kPairChunks;
    if (site_image_needed(c, L))
      pair_loop_f32<S, C0, true>(d, c, k32, li, nt, tile_size, nfar, nnear, p0, p1, acc);
    else
      pair_loop_f32<S, C0, false>(d, c, k32, li, nt, tile_size, nfar, nnear, p0, p1, acc);
  }
  __syncthreads();
  if (ch != 0) return;   // chunk-0 threads (whole warps) finish the molecules
  IAcc a;
  zero_acc(a);
  double wall_e = 0.0;
  if (i < t.count) {
    auto sum = [&](int f) {
      double v = 0.0;
      for (int k = 0; k < kPairChunks; k++) v += acc[f * B + i + k * tile_size];
      return v;
    };
#pragma unroll
    for (int k = 0; k < S; k++)
      for (int x = 0; x < 3; x++) a.fs[k][x] = sum(3 * k + x);
    for (int x = 0; x < 3; x++) {
      a.fc[x] = sum(3 * S + x);
      a.vir[x] = sum(3 * S + 3 + x);
    }
    a.lj = sum(3 * S + 6);
    a.clmb = sum(3 * S + 7);
    a.npair = npairs;
    finish_molecule<S>(d, c, g, L, a, wall_e);
  }
  write_part2(d, c, t, a, wall_e);
}

// FP64 form: one launch per step after the replica head (list rebuild when
// due, pairs, wall, A2M); the box and the rebuild decision come from
// k_replica_head.
__global__ void __launch_bounds__(128, 1) k_force_f64(DevPtrs d, const RepState* __restrict__ X, int tile_size) {
  step_kernel_entry();
  extern __shared__ uint32_t bm[];
  __shared__ double Ls[3];
  __shared__ int rb;
  const int tix = d.order ? d.order[blockIdx.x] : d.tile0 + blockIdx.x;   // costliest tiles first
  const Tile t = d.tiles[tix];
  const RepConst& c = d.rc[t.rep];
  if (threadIdx.x < 3) Ls[threadIdx.x] = X[t.rep].L[threadIdx.x];
  if (threadIdx.x == 0) rb = d.cgrid[t.rep].rebuild;
  __syncthreads();
  const double L[3] = {Ls[0], Ls[1], Ls[2]};
  if (c.nsite == 3)
    force_tile_f64<3, 0>(d, c, t, tix, L, rb != 0, tile_size, bm, d.bm_win);
  else if (c.nsite == 4)
    force_tile_f64<4, 1>(d, c, t, tix, L, rb != 0, tile_size, bm, d.bm_win);
  else
    force_tile_f64<5, 1>(d, c, t, tix, L, rb != 0, tile_size, bm, d.bm_win);
}

// FP32 form, first launch after the replica head: skin-list rebuild when due,
// pass 1; kListLanes x tile threads, the lanes of a molecule adjacent in a
// warp.  Light on registers, so many warps hide the gathered loads.
__global__ void __launch_bounds__(256, 4) k_force_lists(DevPtrs d, const RepState* __restrict__ X, int tile_size) {
  step_kernel_entry();
  extern __shared__ uint32_t bm[];
  __shared__ double Ls[3];
  __shared__ int rb;
  const int tix = d.order ? d.order[blockIdx.x] : d.tile0 + blockIdx.x;
  const Tile t = d.tiles[tix];
  const RepConst& c = d.rc[t.rep];
  if (threadIdx.x < 3) Ls[threadIdx.x] = X[t.rep].L[threadIdx.x];
  if (threadIdx.x == 0) rb = d.cgrid[t.rep].rebuild;
  __syncthreads();
  const double L[3] = {Ls[0], Ls[1], Ls[2]};
  const int i = threadIdx.x / kListLanes, sub = threadIdx.x % kListLanes;
  const int li = t.start + i;
  const bool valid = i < t.count;
  uint16_t* nb = d.nbr + c.nbr_off + (long long)(tix - c.tile_off) * c.nbr_cap * tile_size + i;
  int cnt;
  if (rb) {
    cnt = build_lists_f32(d, c, t, L, nb, tile_size, bm, d.bm_win);
    if (valid && sub == 0) {
      const int* w = reinterpret_cast<const int*>(d.pack) + c.pack_off + (long long)li * c.pack_stride;
      d.ref_com[c.mol_off + li] = make_int4(w[0], w[1], w[2], 0);
    }
    if (threadIdx.x == 0)
      for (int x = 0; x < 3; x++) d.Lbuild[3 * tix + x] = L[x];
    __syncthreads();   // the group's list entries, written by all its lanes, are read below
  } else {
    cnt = valid ? d.nbr_cnt[c.mol_off + li] : 0;
  }
  if (!valid) cnt = 0;
  uint16_t* nt = d.nbt + (nb - d.nbr);
  if (site_image_needed(c, L)) tight_lists_f32<true>(d, c, li, valid, sub, L, nb, nt, cnt, tile_size);
  else tight_lists_f32<false>(d, c, li, valid, sub, L, nb, nt, cnt, tile_size);
}

// FP32 form, second launch of a step: pair forces, wall, A2M (box from X, which
// k_force_lists has updated); kPairChunks x tile threads.
__global__ void __launch_bounds__(128, 3) k_force_pairs(DevPtrs d, const RepState* __restrict__ X,
                                                        int tile_size) {
  step_kernel_entry();
  __shared__ double Ls[3];
  const int tix = d.order ? d.order[blockIdx.x] : d.tile0 + blockIdx.x;
  const Tile t = d.tiles[tix];
  const RepConst& c = d.rc[t.rep];
  if (threadIdx.x < 3) Ls[threadIdx.x] = X[t.rep].L[threadIdx.x];
  __syncthreads();
  const double L[3] = {Ls[0], Ls[1], Ls[2]};
  if (c.nsite == 3)
    force_tile_f32<3, 0>(d, c, t, tix, L, tile_size);
  else if (c.nsite == 4)
    force_tile_f32<4, 1>(d, c, t, tix, L, tile_size);
  else
    force_tile_f32<5, 1>(d, c, t, tix, L, tile_size);
}

// ------------------------------------------------------------------ per-replica kernels

__device__ inline double barostat_energy(const RepConst& c, const RepState& st) {
  // Molecules::BarostatEnergy (src/molecules.cxx:663-678); slit src/remdgpu.cu:2803-2809
  if (c.pconstant > 0) {
    if (c.confined == 0)
      return 0.5 * (st.Pv[0] * st.Pv[0] + st.Pv[1] * st.Pv[1] + st.Pv[2] * st.Pv[2]) / c.W +
             st.P * st.L[0] * st.L[1] * st.L[2];
    if (c.confined == 1) return 0.5 * st.Pv[2] * st.Pv[2] / c.W + st.P * volume(c, st);
    return (st.Pv[0] * st.Pv[0] + st.Pv[1] * st.Pv[1]) * (0.5 / c.W) + st.P * volume(c, st);
  }
  return 0.0;
}

// Molecules::CalcProperties (src/molecules.cxx:702-734) from the reduced kinetic
// sums; writes the REMDGPU::GetAverages fields (T and pressures reduced).
__device__ inline double calc_properties(const DevPtrs& d, const RepConst& c, const RepState& st,
                                         const double* tra3raw, double rot, double* avg, const P2Sum& e) {
  const double lj = e.lj, clmb = e.clmb, wall = e.wall;
  const double* vir = e.vir;
  const double pot = lj + clmb + wall;
  double tmp[3];
  for (int x = 0; x < 3; x++) {
    const double cf = 1.0 / (st.L[x] * st.s);
    tmp[x] = tra3raw[x] * (cf * cf * 0.5);
  }
  const double tra = tmp[0] + tmp[1] + tmp[2];
  const double kin = tra + rot;
  const double tsm = 0.5 * st.Ps * st.Ps / c.Q;
  const double tsp = st.gkT * log(st.s);
  double tot = pot + kin;
  if (c.tconstant == 1) tot += tsm + tsp;
  if (c.pconstant > 0) tot += barostat_energy(c, st);
  const double V = volume(c, st);
  if (avg) {
    avg[0] = lj; avg[1] = clmb; avg[2] = wall; avg[3] = V;
    avg[4] = tra; avg[5] = rot; avg[6] = kin / (3.0 * c.nmol);
    avg[8] = (tmp[0] * 2.0 + vir[0]) / V;
    avg[9] = (tmp[1] * 2.0 + vir[1]) / V;
    avg[10] = (tmp[2] * 2.0 + vir[2]) / V;
    avg[7] = ((tmp[0] * 2.0 + vir[0]) + (tmp[1] * 2.0 + vir[1]) + (tmp[2] * 2.0 + vir[2])) / (3. * V);
    avg[11] = tot; avg[12] = tot - st.H0;
    avg[13] = st.s; avg[14] = st.Ps;
    avg[15] = st.Pv[0]; avg[16] = st.Pv[1]; avg[17] = st.Pv[2]; avg[18] = 0.0;
  }
  return tot;
}

__device__ inline void kinetic_sums(const DevPtrs& d, const RepConst& c, double s, double* acc) {
  const int N = d.N;
  acc[0] = acc[1] = acc[2] = acc[3] = 0.0;
  for (int li = threadIdx.x; li < c.nmol; li += blockDim.x) {
    const int g = c.mol_off + li;
    double q[4], p[4];
    for (int x = 0; x < 4; x++) { q[x] = d.q[x * N + g]; p[x] = d.p[x * N + g]; }
    for (int x = 0; x < 3; x++) {
      const double v = d.v[x * N + g];
      acc[x] += (v * v) * c.mass;
    }
    acc[3] += rot_energy(q, p, c.I, s);
  }
}

__device__ inline void finish_replica(const DevPtrs& d, const RepConst& c, int rep, const RepState& st) {
  double* avg = d.avg + (long long)rep * kNumAvg;
  bool ok = true;
  for (int k = 0; k < kNumAvg; k++) ok = ok && isfinite(avg[k]);
  if (!ok) {
    atomicOr(d.err, kErrNonFinite);
    atomicMax(&d.status[rep], 4);
  }
}

__global__ void __launch_bounds__(kRepThreads) k_replica_end(DevPtrs d, RepState* X) {
  __shared__ RepState st;
  __shared__ double cv[4];
  __shared__ double red[8 * 4];
  const int rep = blockIdx.x;
  const RepConst& c = d.rc[rep];
  P2Sum e;
  if (threadIdx.x < 32) e = reduce_part2(d, c);
  if (threadIdx.x == 0) {
    RepState s = X[rep];
    for (int x = 0; x < 3; x++) cv[x] = s.L[x] * s.s * c.dthalf;
    cv[3] = 2.0 * s.s * c.dthalf;
    d5_scalar(c, s, e.lj + e.clmb + e.wall, e.vir);
    d6(c, s);
    st = s;
  }
  __syncthreads();
  const int N = d.N;
  for (int li = threadIdx.x; li < c.nmol; li += blockDim.x) {
    const int g = c.mol_off + li;
    double v[3], p[4], q[4], f[3], n[4];
    for (int x = 0; x < 3; x++) { v[x] = d.v[x * N + g]; f[x] = d.f[x * N + g]; }
    for (int x = 0; x < 4; x++) { q[x] = d.q[x * N + g]; p[x] = d.p[x * N + g]; n[x] = d.n[x * N + g]; }
    kick(v, p, q, f, n, cv, cv[3], c.mass);
    for (int x = 0; x < 3; x++) d.v[x * N + g] = v[x];
    for (int x = 0; x < 4; x++) d.p[x * N + g] = p[x];
  }
  __syncthreads();
  double acc[4];
  kinetic_sums(d, c, st.s, acc);
  block_sum<4>(acc, red);
  if (threadIdx.x == 0) {
    calc_properties(d, c, st, acc, acc[3], d.avg + (long long)rep * kNumAvg, e);
    X[rep] = st;
    finish_replica(d, c, rep, st);
  }
}

// Initial properties after the first force call: gkT, CalcProperties, H0 = tot
// (Molecules::InitializeProperty, src/molecules.h:260-270).
__global__ void __launch_bounds__(kRepThreads) k_replica_props(DevPtrs d, RepState* X) {
  __shared__ double red[8 * 4];
  const int rep = blockIdx.x;
  const RepConst& c = d.rc[rep];
  RepState st = X[rep];
  double acc[4];
  kinetic_sums(d, c, st.s, acc);
  block_sum<4>(acc, red);
  P2Sum e;
  if (threadIdx.x < 32) e = reduce_part2(d, c);
  if (threadIdx.x == 0) {
    st.gkT = 6.0 * (double)c.nmol * st.T;
    double* avg = d.avg + (long long)rep * kNumAvg;
    st.H0 = calc_properties(d, c, st, acc, acc[3], avg, e);
    avg[12] = 0.0;
    X[rep] = st;
  }
}

// Molecules::KillAngularMomentumInTube (src/molecules.cxx:189-210) for the
// replica of this block: the mean angular momentum about the tube axis, taken
// out of molecules further than 1 A from it; L and s from st.
__device__ void kill_tube_angular_block(const DevPtrs& d, const RepConst& c, const RepState& st,
                                        double* red) {
  const int N = d.N;
  double am[4] = {0, 0, 0, 0};
  for (int li = threadIdx.x; li < c.nmol; li += blockDim.x) {
    const int g = c.mol_off + li;
    double r[3], v[3];
    for (int x = 0; x < 3; x++) {
      r[x] = (d.r[x * N + g] - 0.5) * st.L[x];
      v[x] = d.v[x * N + g] / (st.L[x] * st.s);
    }
    am[0] += c.mass * (r[0] * v[1] - r[1] * v[0]);
    am[1] += c.mass;
  }
  block_sum<4>(am, red);
  const double lz = am[0] / am[1];
  for (int li = threadIdx.x; li < c.nmol; li += blockDim.x) {
    const int g = c.mol_off + li;
    double r[3];
    for (int x = 0; x < 3; x++) r[x] = (d.r[x * N + g] - 0.5) * st.L[x];
    const double r02 = r[0] * r[0] + r[1] * r[1];
    if (r02 > 1.0) {
      d.v[g] += lz * r[1] / r02 * st.L[0] * st.s;
      d.v[N + g] -= lz * r[0] / r02 * st.L[1] * st.s;
    }
  }
  __syncthreads();
}

// Molecules::KillMomentum (src/molecules.cxx:168-187) for the replica of this
// block: the mean momentum removed along the unconfined directions; in a tube
// (z only) it also removes the angular momentum about the axis.
__device__ void kill_momentum_block(const DevPtrs& d, const RepConst& c, const RepState& st,
                                    double* red) {
  const int N = d.N;
  double acc[4] = {0, 0, 0, 0};
  for (int li = threadIdx.x; li < c.nmol; li += blockDim.x) {
    const int g = c.mol_off + li;
    for (int x = 0; x < 3; x++) acc[x] += d.v[x * N + g] * c.mass;
    acc[3] += c.mass;
  }
  block_sum<4>(acc, red);
  const double mom[3] = {acc[0] / acc[3], acc[1] / acc[3], acc[2] / acc[3]};
  for (int li = threadIdx.x; li < c.nmol; li += blockDim.x) {
    const int g = c.mol_off + li;
    if (c.confined == 1) {
      d.v[2 * N + g] -= mom[2];
    } else if (c.confined == 2) {
      d.v[g] -= mom[0];
      d.v[N + g] -= mom[1];
    } else {
      for (int x = 0; x < 3; x++) d.v[x * N + g] -= mom[x];
    }
  }
  __syncthreads();
  if (c.confined == 1) kill_tube_angular_block(d, c, st, red);
}

// The exchange tail for a replica whose condition changed (src/remd.cxx:526-536):
// ChangeTemperature (src/molecules.h:333-353), KillMomentum (+ the tube's angular
// momentum, src/molecules.cxx:168-210), SetPressure, CalcProperties, UpdateHamiltonian.
__global__ void __launch_bounds__(kRepThreads) k_replica_start(DevPtrs d, RepState* X) {
  __shared__ RepState st;
  __shared__ double sh[4];
  __shared__ double red[8 * 4];
  const int rep = blockIdx.x;
  const RepConst& c = d.rc[rep];
  const double Tn = d.newT[rep], Pn = d.newP[rep];
  {
    const RepState s0 = X[rep];
    if (Tn == s0.T && Pn == s0.P) return;   // uniform over the block
  }
  if (threadIdx.x == 0) {
    RepState s = X[rep];
    const double coef = sqrt(Tn / s.T);
    sh[0] = coef / s.s;
    s.Ps *= coef;
    if (c.pconstant == 1) s.Pv[0] *= coef * s.s;
    if (c.pconstant == 2) s.Pv[2] *= coef * s.s;
    if (c.pconstant == 3) { s.Pv[0] *= coef * s.s; s.Pv[1] *= coef * s.s; }
    s.T = Tn;
    s.gkT = 6.0 * (double)c.nmol * s.T;
    s.s = 1.0;
    st = s;
  }
  __syncthreads();
  const int N = d.N;
  const double sc = sh[0];
  for (int li = threadIdx.x; li < c.nmol; li += blockDim.x) {
    const int g = c.mol_off + li;
    for (int x = 0; x < 3; x++) d.v[x * N + g] *= sc;
    for (int x = 0; x < 4; x++) d.p[x * N + g] *= sc;
  }
  __syncthreads();
  kill_momentum_block(d, c, st, red);
  double kacc[4];
  kinetic_sums(d, c, st.s, kacc);
  block_sum<4>(kacc, red);
  P2Sum e;
  if (threadIdx.x < 32) e = reduce_part2(d, c);
  if (threadIdx.x == 0) {
    RepState s = st;
    s.P = Pn;
    s.H0 = calc_properties(d, c, s, kacc, kacc[3], nullptr, e);
    X[rep] = s;
  }
}

// Molecules::VelocityScaling + AngVelocityScaling (src/molecules.cxx:261-311):
// translational and rotational kinetic energies set to 1.5 N T each, momentum
// removed (along z plus the angular momentum about the axis in a tube),
// thermostat and barostat momenta reset.
//  PER_STEP = false: the reference's init_scaling, after which H0 is recomputed
//    (InitializeProperty).  The stored v and p carry a factor s; they are first
//    brought to s = 1 (the reference calls this only at start-up, where s = 1
//    already, and resetting s afterwards would otherwise scale the kinetic
//    energy by 1/s^2).
//  PER_STEP = true: the velocity-scaling thermostat (tconstant 2) before every
//    MD step, for those replicas only, in the reference's exact order (kinetic
//    energy with the current s, then s = 1, then the rotational part); H0 and
//    the averages are left alone.
template <bool PER_STEP>
__global__ void __launch_bounds__(kRepThreads) k_replica_rescale(DevPtrs d, RepState* X) {
  __shared__ RepState st;
  __shared__ double red[8 * 4];
  const int rep = blockIdx.x;
  const RepConst& c = d.rc[rep];
  if (PER_STEP && c.tconstant != 2) return;   // uniform for the block
  if (threadIdx.x == 0) st = X[rep];
  __syncthreads();
  const int N = d.N;
  if (!PER_STEP && st.s != 1.0) {
    const double si = 1.0 / st.s;
    for (int li = threadIdx.x; li < c.nmol; li += blockDim.x) {
      const int g = c.mol_off + li;
      for (int x = 0; x < 3; x++) d.v[x * N + g] *= si;
      for (int x = 0; x < 4; x++) d.p[x * N + g] *= si;
    }
    __syncthreads();
    if (threadIdx.x == 0) st.s = 1.0;
    __syncthreads();
  }
  double k[4];
  kinetic_sums(d, c, st.s, k);
  block_sum<4>(k, red);
  {
    double tra = 0.0;
    for (int x = 0; x < 3; x++) {
      const double cf = 1.0 / (st.L[x] * st.s);
      tra += k[x] * (cf * cf * 0.5);
    }
    const double coef = (tra > 0.0) ? sqrt(1.5 * c.nmol * st.T / tra) : 1.0;
    for (int li = threadIdx.x; li < c.nmol; li += blockDim.x)
      for (int x = 0; x < 3; x++) d.v[x * N + c.mol_off + li] *= coef;
  }
  __syncthreads();
  kill_momentum_block(d, c, st, red);
  // VelocityScaling takes the tube's angular momentum out once more after KillMomentum
  if (c.confined == 1) kill_tube_angular_block(d, c, st, red);
  __syncthreads();
  if (threadIdx.x == 0) {
    st.s = 1.0;
    st.Ps = 0.0;
    st.Pv[0] = st.Pv[1] = st.Pv[2] = 0.0;
  }
  __syncthreads();
  kinetic_sums(d, c, st.s, k);
  block_sum<4>(k, red);
  {
    const double coef = (k[3] > 0.0) ? sqrt(1.5 * c.nmol * st.T / k[3]) : 1.0;
    for (int li = threadIdx.x; li < c.nmol; li += blockDim.x)
      for (int x = 0; x < 4; x++) d.p[x * N + c.mol_off + li] *= coef;
  }
  __syncthreads();
  if (PER_STEP) {
    if (threadIdx.x == 0) X[rep] = st;
    return;
  }
  kinetic_sums(d, c, st.s, k);
  block_sum<4>(k, red);
  P2Sum e;
  if (threadIdx.x < 32) e = reduce_part2(d, c);
  if (threadIdx.x == 0) {
    RepState s = st;
    s.gkT = 6.0 * (double)c.nmol * s.T;
    double* avg = d.avg + (long long)rep * kNumAvg;
    s.H0 = calc_properties(d, c, s, k, k[3], avg, e);
    avg[12] = 0.0;
    X[rep] = s;
  }
}

// ------------------------------------------------------------------ exchange
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): a counter-based generator.
__device__ inline uint4 philox4x32(uint4 ctr, uint2 key) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  for (int i = 0; i < 10; i++) {
    const uint32_t hi0 = __umulhi(M0, ctr.x), lo0 = M0 * ctr.x;
    const uint32_t hi1 = __umulhi(M1, ctr.z), lo1 = M1 * ctr.z;
    ctr = make_uint4(hi1 ^ ctr.y ^ key.x, lo1, hi0 ^ ctr.w ^ key.y, lo0);
    key.x += W0;
    key.y += W1;
  }
  return ctr;
}

__device__ inline double philox_uniform(unsigned long long seed, long step, int ens, int pair) {
  const uint4 r = philox4x32(make_uint4((uint32_t)pair, (uint32_t)ens, (uint32_t)step,
                                        (uint32_t)((unsigned long long)step >> 32)),
                             make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
  const unsigned long long b = ((unsigned long long)r.x << 32 | r.y) >> 11;
  return (double)b * (1.0 / 9007199254740992.0);
}

// REMD::ReplicaExchange + ExchangeList (src/remd.cxx:467-538, src/remdinfo.cxx:54-125),
// one thread per ensemble; pot/vol from the averages of the last interval.
// step < 0: the ensemble's own interval counter (step_ctr[e]) is used and then
// advanced, and the uniforms come from Philox -- the form captured in the
// interval graph.
__global__ void k_exchange(DevPtrs d, const int* grid, const int* rep_off, const int* u_off,
                           int nens, long step_arg, const double* u, const unsigned long long* seeds,
                           int* index, double* T, double* P, long long* step_ctr) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nens) return;
  long step = step_arg;
  if (step_arg < 0) {
    step = (long)step_ctr[e];
    step_ctr[e] = step + 1;
  }
  const int nt = grid[2 * e], np = grid[2 * e + 1];
  const int off = rep_off[e];
  const int pcon = d.rc[off].pconstant;
  const int ec = (int)(step % 4);
  int* idx = index + off;
  double* Te = T + off;
  double* Pe = P + off;
  auto pot_of = [&](int r) {
    const double* a = d.avg + (long long)(off + r) * kNumAvg;
    return a[0] + a[1] + a[2];
  };
  auto vol_of = [&](int r) { return d.avg[(long long)(off + r) * kNumAvg + 3]; };
  int pair = 0;
  auto trial = [&](int a, int b) {
    const int i1 = idx[a], i2 = idx[b];
    const double b1 = 1. / Te[i1], b2 = 1. / Te[i2];
    double delta = (b2 - b1) * (pot_of(i1) - pot_of(i2));
    if (pcon > 0) delta += (b2 * Pe[i2] - b1 * Pe[i1]) * (vol_of(i1) - vol_of(i2));
    const double uu = u ? u[u_off[e] + pair] : philox_uniform(seeds[e], step, 0, pair);
    pair++;
    if (exp(-delta) > uu) {
      double t = Te[idx[a]]; Te[idx[a]] = Te[idx[b]]; Te[idx[b]] = t;
      t = Pe[idx[a]]; Pe[idx[a]] = Pe[idx[b]]; Pe[idx[b]] = t;
      const int ti = idx[a]; idx[a] = idx[b]; idx[b] = ti;
    }
  };
  if (ec == 0) {
    for (int j = 0; j < np; ++j)
      for (int i = 0; i < nt / 2; ++i) trial(2 * i + j * nt, 2 * i + 1 + j * nt);
  } else if (ec == 1) {
    for (int j = 0; j < np / 2; ++j)
      for (int i = 0; i < nt; ++i) trial(i + 2 * j * nt, i + (2 * j + 1) * nt);
  } else if (ec == 2) {
    for (int j = 0; j < np; ++j)
      for (int i = 0; i < nt / 2 - (nt + 1) % 2; ++i) trial(2 * i + j * nt + 1, 2 * i + 1 + j * nt + 1);
  } else {
    for (int j = 0; j < np / 2 - (np + 1) % 2; ++j)
      for (int i = 0; i < nt; ++i) trial(i + (2 * j + 1) * nt, i + (2 * j + 2) * nt);
  }
}

// ------------------------------------------------------------------ FP32 peak probe
// Eight independent FMA chains per thread, register resident: measures the
// FP32 pipe's FMA throughput (the force kernel's roofline denominator).
__global__ void __launch_bounds__(256) k_fma_peak(float* out, int iters, float a, float b) {
  float x0 = threadIdx.x * 1e-3f, x1 = x0 + 1.f, x2 = x0 + 2.f, x3 = x0 + 3.f;
  float x4 = x0 + 4.f, x5 = x0 + 5.f, x6 = x0 + 6.f, x7 = x0 + 7.f;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 16; k++) {
      x0 = fmaf(x0, a, b); x1 = fmaf(x1, a, b); x2 = fmaf(x2, a, b); x3 = fmaf(x3, a, b);
      x4 = fmaf(x4, a, b); x5 = fmaf(x5, a, b); x6 = fmaf(x6, a, b); x7 = fmaf(x7, a, b);
    }
  }
  const float s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
  if (s == 12345.678f) out[blockIdx.x] = s;   // keeps the chains live
}

int measure_fp32_fma(int device, double* ms, long long* flops) {
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return 6;
  const int blocks = prop.multiProcessorCount * 8, threads = 256, iters = 4096;
  float* out = nullptr;
  if (cudaMalloc(&out, blocks * sizeof(float)) != cudaSuccess) return 2;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  k_fma_peak<<<blocks, threads>>>(out, 64, 0.999f, 1e-3f);   // warm-up
  float best = 1e30f;
  for (int rep = 0; rep < 5; rep++) {
    cudaEventRecord(e0);
    k_fma_peak<<<blocks, threads>>>(out, iters, 0.999f, 1e-3f);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    best = fminf(best, t);
  }
  const cudaError_t err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (err != cudaSuccess) return 6;
  *ms = best;
  *flops = (long long)blocks * threads * iters * 16LL * 8LL * 2LL;
  return 0;
}

// Throughput of integer adds into shared memory (64- and 32-bit), into a peer
// block's shared memory (clusters of four) and into global memory (L2): the
// rates at which a pair kernel that computes each pair once could add the
// partner molecule's share of the forces.  Fixed-point sums do not depend on
// the order of their terms, so such a kernel would stay deterministic.  Each
// thread adds to pseudo-random words of a per-block array of kAtomWords words
// (7 values x 736 molecules); every index is taken modulo that size.
constexpr int kAtomWords = 7 * 736;
constexpr int kAtomThreads = 512, kAtomBlocksPerSM = 4, kAtomIters = 4096;

__device__ __forceinline__ unsigned atom_hash(unsigned x) {
  x ^= x >> 16; x *= 0x7feb352dU; x ^= x >> 15; x *= 0x846ca68bU; x ^= x >> 16;
  return x;
}

template <int MODE>   // 0 shared u64, 1 shared u32, 2 u64 into cluster peers, 3 global u64
__global__ void __launch_bounds__(kAtomThreads) k_atomic_rate(unsigned long long* gbuf, unsigned long long* out,
                                                              int iters) {
  extern __shared__ unsigned long long ash[];
  for (int k = threadIdx.x; k < kAtomWords; k += blockDim.x) ash[k] = 0ull;
  if (MODE == 2) cg::this_cluster().sync(); else __syncthreads();
  unsigned long long* g = gbuf + (size_t)blockIdx.x * kAtomWords;
  unsigned s = atom_hash(threadIdx.x * 7919u + blockIdx.x * 104729u);
  for (int it = 0; it < iters; it++) {
    s = atom_hash(s + (unsigned)it);
    const int idx = (int)(s % (unsigned)kAtomWords);
    if (MODE == 0) atomicAdd(&ash[idx], (unsigned long long)(s & 1023u));
    if (MODE == 1) atomicAdd(reinterpret_cast<unsigned*>(ash) + idx, s & 1023u);
    if (MODE == 2) atomicAdd(cg::this_cluster().map_shared_rank(ash, (int)((s >> 20) & 3u)) + idx,
                             (unsigned long long)(s & 1023u));
    if (MODE == 3) atomicAdd(g + idx, (unsigned long long)(s & 1023u));
  }
  // a cluster's blocks leave only when no peer adds into their memory any more
  if (MODE == 2) cg::this_cluster().sync(); else __syncthreads();
  unsigned long long t = 0ull;
  for (int k = threadIdx.x; k < kAtomWords; k += blockDim.x) t += ash[k];
  if (t == 0x5eedull) atomicAdd(out, t);   // keeps the adds live
}

int measure_atomics(int device, double* rates) {
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return 6;
  const int blocks = prop.multiProcessorCount * kAtomBlocksPerSM;   // 148 SMs: a multiple of 4
  if (blocks % 4) return 6;
  const size_t smem = kAtomWords * sizeof(unsigned long long);
  unsigned long long *g = nullptr, *out = nullptr;
  if (cudaMalloc(&g, (size_t)blocks * smem) != cudaSuccess) return 2;
  if (cudaMalloc(&out, 8) != cudaSuccess) { cudaFree(g); return 2; }
  cudaMemset(g, 0, (size_t)blocks * smem);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  auto launch = [&](int mode, int iters) {
    if (mode == 2) {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(blocks);
      cfg.blockDim = dim3(kAtomThreads);
      cfg.dynamicSmemBytes = smem;
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeClusterDimension;
      at[0].val.clusterDim.x = 4;
      at[0].val.clusterDim.y = 1;
      at[0].val.clusterDim.z = 1;
      cfg.attrs = at;
      cfg.numAttrs = 1;
      cudaLaunchKernelEx(&cfg, k_atomic_rate<2>, g, out, iters);
    } else if (mode == 0) {
      k_atomic_rate<0><<<blocks, kAtomThreads, smem>>>(g, out, iters);
    } else if (mode == 1) {
      k_atomic_rate<1><<<blocks, kAtomThreads, smem>>>(g, out, iters);
    } else {
      k_atomic_rate<3><<<blocks, kAtomThreads, smem>>>(g, out, iters);
    }
  };
  for (int mode = 0; mode < 4; mode++) {
    launch(mode, 64);   // warm-up
    float best = 1e30f;
    for (int rep = 0; rep < 3; rep++) {
      cudaEventRecord(e0);
      launch(mode, kAtomIters);
      cudaEventRecord(e1);
      cudaEventSynchronize(e1);
      float t = 0.f;
      cudaEventElapsedTime(&t, e0, e1);
      best = fminf(best, t);
    }
    rates[mode] = (double)blocks * kAtomThreads * kAtomIters / (best * 1e-3) / 1e9;
  }
  const cudaError_t err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(g);
  cudaFree(out);
  return err == cudaSuccess ? 0 : 6;
}

// ------------------------------------------------------------------ caller-buffer variant
// Entry and exit kernels of remd_force_snapshot_noalloc (noalloc.cu): the
// caller's AoS positions/quaternions into the scratch SoA arrays and force
// records, and the scratch results back into the caller's AoS outputs.  The
// constants, tiles and box arrive as a kernel parameter; block 0 stores them
// into the scratch for the force kernels that follow on the same stream.
__global__ void k_noalloc_load(DevPtrs d, const NoAllocSetup setup, RepState* __restrict__ X,
                               const double* __restrict__ r_aos, const double* __restrict__ q_aos) {
  const Tile t = setup.tiles[blockIdx.x];
  const RepConst& c = setup.c;
  const int i = threadIdx.x;
  if (i < t.count) {
    const int li = t.start + i;
    const int g = c.mol_off + li;
    double r[3], q[4];
    for (int x = 0; x < 3; x++) r[x] = r_aos[3 * li + x];
    for (int x = 0; x < 4; x++) q[x] = q_aos[4 * li + x];
    for (int x = 0; x < 3; x++) d.r[x * d.N + g] = r[x];
    for (int x = 0; x < 4; x++) d.q[x * d.N + g] = q[x];
    write_pack(d, c, kF32, li, r, q);
  }
  if (i == 0) {
    const double nan = __longlong_as_double(0x7ff8000000000000ll);
    d.Lbuild[3 * blockIdx.x] = nan;
    if (blockIdx.x == 0) {
      *const_cast<RepConst*>(d.rc) = setup.c;
      for (int k = 0; k < d.ntiles; k++) const_cast<Tile*>(d.tiles)[k] = setup.tiles[k];
      *X = setup.rs;
      *d.err = 0;
      d.status[0] = 0;
    }
  }
}

// out: lj, clmb, wall, vir[3] (halved like ForceCalculator::Switching), the
// number of unordered pairs within rcut, and the error word (0 = ok).
__global__ void k_noalloc_store(DevPtrs d, double* __restrict__ f_aos, double* __restrict__ n_aos,
                                double* __restrict__ out) {
  const RepConst& c = d.rc[0];
  for (int li = threadIdx.x; li < c.nmol; li += blockDim.x) {
    const int g = c.mol_off + li;
    for (int x = 0; x < 3; x++) f_aos[3 * li + x] = d.f[x * d.N + g];
    for (int x = 0; x < 4; x++) n_aos[4 * li + x] = d.n[x * d.N + g];
  }
  P2Sum e;
  if (threadIdx.x < 32) e = reduce_part2(d, c);
  if (threadIdx.x == 0) {
    long long np = 0;
    for (int t = c.warp_off; t < c.warp_off + c.nwarp; t++) np += d.part2[t].npairs;
    out[0] = e.lj; out[1] = e.clmb; out[2] = e.wall;
    out[3] = e.vir[0]; out[4] = e.vir[1]; out[5] = e.vir[2];
    out[6] = (double)(np / 2);
    out[7] = (double)*d.err;
  }
}

void launch_noalloc_load(const DevPtrs& d, const NoAllocSetup& setup, RepState* X, const double* r_aos,
                         const double* q_aos, int tile, cudaStream_t s) {
  k_noalloc_load<<<d.ntiles, tile, 0, s>>>(d, setup, X, r_aos, q_aos);
}
void launch_noalloc_store(const DevPtrs& d, double* f_aos, double* n_aos, double* out, cudaStream_t s) {
  k_noalloc_store<<<1, 256, 0, s>>>(d, f_aos, n_aos, out);
}

// ------------------------------------------------------------------ carrying replicas between handles
// The serving loop's batch changes: replicas that keep running are copied from
// the previous handle's arrays into the new handle's, on the device.
// src[k] = {first molecule of replica k in the old arrays, old replica} or -1.
__global__ void k_carry_molecules(DevPtrs d, const double* __restrict__ r, const double* __restrict__ v,
                                  const double* __restrict__ q, const double* __restrict__ p, int No,
                                  const int2* __restrict__ src) {
  const Tile t = d.tiles[blockIdx.x];
  const int so = src[t.rep].x;
  const int i = threadIdx.x;
  if (so < 0 || i >= t.count) return;
  const int li = t.start + i;
  const int g = d.rc[t.rep].mol_off + li, go = so + li;
  const int N = d.N;
  for (int x = 0; x < 3; x++) {
    d.r[x * N + g] = r[(long long)x * No + go];
    d.v[x * N + g] = v[(long long)x * No + go];
  }
  for (int x = 0; x < 4; x++) {
    d.q[x * N + g] = q[(long long)x * No + go];
    d.p[x * N + g] = p[(long long)x * No + go];
  }
}

// Per replica: the scalars and the pending condition; per ensemble (sens[e] =
// old ensemble or -1): the exchange's slot -> replica index, interval counter
// and seed.
__global__ void k_carry_replicas(int nrep, int nens, RepState* __restrict__ X, const RepState* __restrict__ Xo,
                                 double* __restrict__ T, double* __restrict__ P, const double* __restrict__ To,
                                 const double* __restrict__ Po, const int2* __restrict__ src,
                                 const int* __restrict__ sens, const int* __restrict__ rep_off,
                                 const int* __restrict__ rep_off_o, const int* __restrict__ nrep_e,
                                 int* __restrict__ index, const int* __restrict__ index_o,
                                 long long* __restrict__ step, const long long* __restrict__ step_o,
                                 unsigned long long* __restrict__ seed,
                                 const unsigned long long* __restrict__ seed_o) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nrep; k += gridDim.x * blockDim.x) {
    const int so = src[k].y;
    if (so < 0) continue;
    X[k] = Xo[so];
    T[k] = To[so];
    P[k] = Po[so];
  }
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nens; e += gridDim.x * blockDim.x) {
    const int eo = sens[e];
    if (eo < 0) continue;
    for (int c = 0; c < nrep_e[e]; c++) index[rep_off[e] + c] = index_o[rep_off_o[eo] + c];
    step[e] = step_o[eo];
    seed[e] = seed_o[eo];
  }
}

void launch_carry(const DevPtrs& d, const DevPtrs& o, int tile, const int2* src, RepState* X, const RepState* Xo,
                  double* T, double* P, const double* To, const double* Po, int nens, const int* sens,
                  const int* rep_off, const int* rep_off_o, const int* nrep_e, int* index, const int* index_o,
                  long long* step, const long long* step_o, unsigned long long* seed,
                  const unsigned long long* seed_o, bool molecules, cudaStream_t s) {
  if (molecules) k_carry_molecules<<<d.ntiles, tile, 0, s>>>(d, o.r, o.v, o.q, o.p, o.N, src);
  k_carry_replicas<<<(std::max(d.nrep, nens) + 127) / 128, 128, 0, s>>>(
      d.nrep, nens, X, Xo, T, P, To, Po, src, sens, rep_off, rep_off_o, nrep_e, index, index_o, step, step_o,
      seed, seed_o);
}

// ------------------------------------------------------------------ launchers
void launch_pack(const DevPtrs& d, int prec, int tile, cudaStream_t s) {
  k_pack<<<d.ntiles, tile, 0, s>>>(d, prec);
}
static int sm_count() {
  static int n[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return 1 << 30;
  if (!n[dev]) cudaDeviceGetAttribute(&n[dev], cudaDevAttrMultiProcessorCount, dev);
  return n[dev];
}

// A step kernel (it calls step_kernel_entry first).  With `pdl` it is launched
// with programmatic stream serialisation.  That pays where a step's tile grid
// is smaller than the GPU (one block per SM or fewer): the launches are
// latency-bound and the early-scheduled blocks wait on otherwise idle SMs
// (16 replicas of 128 TIP4P molecules: 55 -> 58.5 M mol-steps/s).  Where the
// grid fills the GPU, the waiting blocks hold slots that the other chains of
// the interval graph would use (256 replicas, 111 432 molecules: 288 -> 253 M
// with it), so those launches are plain.
template <typename... KArgs, typename... Args>
static void launch_step_kernel(bool pdl, void (*k)(KArgs...), unsigned grid, unsigned block, size_t smem,
                               cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl ? 1 : 0;
  cudaLaunchKernelEx(&cfg, k, args...);
}

void launch_integrate_prec(const DevPtrs& d, const RepState* X, RepState* Y, bool mid, int tile,
                           int prec, cudaStream_t s) {
  const bool pdl = d.ntiles <= sm_count();
  if (mid)
    launch_step_kernel(pdl, k_integrate<true>, d.ntiles, tile, 0, s, d, X, Y, prec);
  else
    launch_step_kernel(pdl, k_integrate<false>, d.ntiles, tile, 0, s, d, X, Y, prec);
}
int max_force_tile(int prec) { return prec == kF32 ? 128 / kPairChunks : 128; }

size_t force_smem_bytes(int tile) { return (size_t)(3 * kMaxSites + 8) * tile * sizeof(double); }

// Bitmap of the list rebuild: one row of (win | 1) words per thread.
size_t bitmap_smem_bytes(int tile, int win) { return (size_t)tile * (size_t)(win | 1) * sizeof(uint32_t); }

int bitmap_window(int max_nmol) { return std::min((max_nmol + 31) / 32, kBitmapMaxWords); }

cudaError_t force_kernel_setup() {
  // FP32 form: dynamic shared memory = the per-thread FP64 accumulators of a tile
  // of up to 128 molecules (23.5 KB, under the default limit; set explicitly so
  // that a larger tile or more accumulators only change force_smem_bytes); the
  // list kernels' rebuild bitmaps (up to 128 rows of kBitmapMaxWords + 1 words)
  cudaError_t e = cudaFuncSetAttribute(k_force_pairs, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)force_smem_bytes(128));
  if (e != cudaSuccess) return e;
  const int bms = (int)bitmap_smem_bytes(128, kBitmapMaxWords);
  e = cudaFuncSetAttribute(k_force_lists, cudaFuncAttributeMaxDynamicSharedMemorySize, bms);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_force_f64, cudaFuncAttributeMaxDynamicSharedMemorySize, bms);
}

// The force launches of one step; e_head / e_lists (may be null) are recorded
// after the head and after the list kernel (profiling: remd_profile_split).
static void launch_force_impl(const DevPtrs& d, const RepState* Yin, RepState* Xout, int prec, bool force_only,
                              int tile, cudaStream_t s, cudaEvent_t e_head, cudaEvent_t e_lists) {
  const RepState* Xc = Xout;
  const bool pdl = d.ntiles <= sm_count();   // the step's tile grid (see launch_step_kernel)
  if (force_only) launch_step_kernel(pdl, k_replica_head<true>, d.nrep_l, kRepThreads, 0, s, d, Yin, Xout);
  else launch_step_kernel(pdl, k_replica_head<false>, d.nrep_l, kRepThreads, 0, s, d, Yin, Xout);
  if (e_head) cudaEventRecord(e_head, s);
  const size_t bms = bitmap_smem_bytes(tile, d.bm_win);
  if (prec == kF32) {
    launch_step_kernel(pdl, k_force_lists, d.ntiles, kListLanes * tile, bms, s, d, Xc, tile);
    if (e_lists) cudaEventRecord(e_lists, s);
    launch_step_kernel(pdl, k_force_pairs, d.ntiles, kPairChunks * tile, force_smem_bytes(kPairChunks * tile), s,
                       d, Xc, tile);
  } else {
    if (e_lists) cudaEventRecord(e_lists, s);
    launch_step_kernel(pdl, k_force_f64, d.ntiles, tile, bms, s, d, Xc, tile);
  }
}

void launch_force(const DevPtrs& d, const RepState* Yin, RepState* Xout, int prec, bool force_only,
                  int tile, cudaStream_t s) {
  launch_force_impl(d, Yin, Xout, prec, force_only, tile, s, nullptr, nullptr);
}

void launch_force_timed(const DevPtrs& d, const RepState* Yin, RepState* Xout, int prec, int tile, cudaStream_t s,
                        cudaEvent_t e_head, cudaEvent_t e_lists) {
  launch_force_impl(d, Yin, Xout, prec, false, tile, s, e_head, e_lists);
}
void launch_replica_start(const DevPtrs& d, RepState* X, cudaStream_t s) {
  k_replica_start<<<d.nrep, kRepThreads, 0, s>>>(d, X);
}
void launch_replica_end(const DevPtrs& d, RepState* X, cudaStream_t s) {
  k_replica_end<<<d.nrep, kRepThreads, 0, s>>>(d, X);
}
void launch_replica_props(const DevPtrs& d, RepState* X, cudaStream_t s) {
  k_replica_props<<<d.nrep, kRepThreads, 0, s>>>(d, X);
}
void launch_replica_rescale(const DevPtrs& d, RepState* X, bool per_step, cudaStream_t s) {
  if (per_step) k_replica_rescale<true><<<d.nrep, kRepThreads, 0, s>>>(d, X);
  else k_replica_rescale<false><<<d.nrep, kRepThreads, 0, s>>>(d, X);
}
// ------------------------------------------------------------------ histograms
// One thread per condition slot k (slot c of ensemble e).  The sample is the
// Average of the replica at that condition, per molecule (src/remd.cxx:806-811):
// p = (LJ + CLMB + WALL) / nmol, v = VOL / nmol.  Binning, range check and the
// occupied-range bookkeeping follow REMDInfo::IncrementHistogram
// (src/remdinfo.h:299-321) and Histogram::Increment (src/remdinfo.cxx:38-51);
// KeepAverages adds the 19 fields to the bin.  A sample outside
// [min, max) -- or one whose bin rounds up to kHistBins -- is not counted and
// sets kErrHistRange (the reference exits there).  Each slot has one writer,
// so no atomics are needed on the bins.
__global__ void k_histogram(DevPtrs d, const HistEns* __restrict__ he, const int* __restrict__ rep_off,
                            const int* __restrict__ index) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.nrep) return;
  const int e = d.rc[k].ens;
  const HistEns H = he[e];
  if (!H.hist) return;
  const int c = k - rep_off[e];
  const int rep = rep_off[e] + index[k];
  const double* a = d.avg + (long long)rep * kNumAvg;
  const double nmol = (double)d.rc[rep].nmol;
  const double pot = (a[0] + a[1] + a[2]) / nmol;
  const double vol = a[3] / nmol;
  bool ok = !(vol < H.vmin || vol >= H.vmax || pot < H.emin || pot >= H.emax);
  const int v = ok ? (int)((vol - H.vmin) / H.dv) : 0;
  const int p = ok ? (int)((pot - H.emin) / H.de) : 0;
  ok = ok && v >= 0 && v < kHistBins && p >= 0 && p < kHistBins;
  if (!ok) {
    atomicOr(d.err, kErrHistRange);
    return;
  }
  int* b = H.bounds + 5 * c;
  if (b[4] == 0) {
    b[0] = b[1] = v;
    b[2] = b[3] = p;
  }
  b[0] = min(b[0], v);
  b[1] = max(b[1], v);
  b[2] = min(b[2], p);
  b[3] = max(b[3], p);
  b[4] += 1;
  const long long bin = ((long long)c * kHistBins + v) * kHistBins + p;
  H.hist[bin] += 1;
  double* s = H.ave + bin * kNumAvg;
  for (int x = 0; x < kNumAvg; x++) s[x] += a[x];
}

void launch_histogram(const DevPtrs& d, const HistEns* he, const int* rep_off, const int* index,
                      cudaStream_t s) {
  k_histogram<<<(d.nrep + 127) / 128, 128, 0, s>>>(d, he, rep_off, index);
}

void launch_exchange_k(const DevPtrs& d, const int* grid, const int* rep_off, const int* u_off,
                       int nens, long step, const double* u, const unsigned long long* seeds,
                       int* index, double* T, double* P, long long* step_ctr, cudaStream_t s) {
  k_exchange<<<(nens + 63) / 64, 64, 0, s>>>(d, grid, rep_off, u_off, nens, step, u, seeds, index, T,
                                             P, step_ctr);
}

}  // namespace remd
