// kernels.cuh -- the engine's CUDA kernels (sm_100a).
//
// One MD step of every replica of every ensemble is a short chain of launches
// (a tile = 32 or 64 consecutive molecules of one replica, up to 128 in the
// FP64 form):
//
//   k_integrate     [end of the previous step: D5 kick, D5/D6 scalars]
//                   D6, D5, D4, D3 D2 D1 D2 D3 (src/integrator.cxx:646-673),
//                   then the force record of every molecule (fixed-point centre
//                   of mass + rotated site offsets) and the partial sums PsPv needs;
//   k_replica_head  per replica: PsPv + D4 (scalar chain), the neighbour-list
//                   decision and, when a rebuild is due, the cell lists;
//   k_force_lists   per tile (FP32, four lanes per molecule): the list rebuild
//                   when due, then the per-step list of the pairs within rcut;
//   k_force_pairs   per tile (FP32): the switched LJ + Coulomb pair loop, the
//                   wall, and the site -> molecule torque (A2M);
//   k_force_f64     per tile (FP64 form): rebuild, pair loop, wall, A2M.
//
// An interval is k_replica_start (exchange tail), interval x (step chain),
// k_replica_end (last D5/D6 + CalcProperties -> Average), captured once as a
// CUDA graph.
#pragma once
#include "engine_types.cuh"

namespace remd {

enum Prec : int { kF32 = 0, kF64 = 1 };

// host-side launchers (kernels.cu)
void launch_pack(const DevPtrs& d, int prec, int tile, cudaStream_t s);
void launch_integrate_prec(const DevPtrs& d, const RepState* X, RepState* Y, bool mid, int tile,
                           int prec, cudaStream_t s);
// Largest force tile (molecules per block) of a precision: FP32 blocks hold two threads per molecule.
int max_force_tile(int prec);
// Kernel attributes the force launches need (call once per device before launching).
cudaError_t force_kernel_setup();
// Words per row of the list-rebuild bitmap for replicas of up to max_nmol molecules (DevPtrs::bm_win).
int bitmap_window(int max_nmol);
void launch_force(const DevPtrs& d, const RepState* Yin, RepState* Xout, int prec, bool force_only,
                  int tile, cudaStream_t s);
// launch_force(..., force_only = false, ...) with events recorded after the
// replica head and after the list kernel (FP64 form: before its one kernel).
void launch_force_timed(const DevPtrs& d, const RepState* Yin, RepState* Xout, int prec, int tile, cudaStream_t s,
                        cudaEvent_t e_head, cudaEvent_t e_lists);
void launch_replica_start(const DevPtrs& d, RepState* X, cudaStream_t s);
void launch_replica_end(const DevPtrs& d, RepState* X, cudaStream_t s);
void launch_replica_props(const DevPtrs& d, RepState* X, cudaStream_t s);
void launch_replica_rescale(const DevPtrs& d, RepState* X, bool per_step, cudaStream_t s);
void launch_exchange_k(const DevPtrs& d, const int* grid, const int* rep_off, const int* u_off,
                       int nens, long step, const double* u, const unsigned long long* seeds,
                       int* index, double* T, double* P, long long* step_ctr, cudaStream_t s);
// REMD::IncrementHistogram (src/remd.cxx:803-813) for every condition slot of the
// ensembles with a histogram; index[slot] = the replica (ensemble-local) there.
void launch_histogram(const DevPtrs& d, const HistEns* he, const int* rep_off, const int* index,
                      cudaStream_t s);
int pack_stride(int nsite, int prec);
// Set-up of one remd_force_snapshot_noalloc call, passed by value to its load
// kernel (kernel parameters, so no host staging buffer has to outlive the call).
constexpr int kNoAllocMaxTiles = 32;
struct NoAllocSetup {
  RepConst c;
  RepState rs;
  Tile tiles[kNoAllocMaxTiles];
};
void launch_noalloc_load(const DevPtrs& d, const NoAllocSetup& setup, RepState* X, const double* r_aos,
                         const double* q_aos, int tile, cudaStream_t s);
void launch_noalloc_store(const DevPtrs& d, double* f_aos, double* n_aos, double* out, cudaStream_t s);
int measure_fp32_fma(int device, double* ms, long long* flops);
int measure_atomics(int device, double* rates);
// Copies carried replicas from handle arrays `o` into `d` (serving batch changes):
// molecule state (when `molecules`), RepState, pending condition, and per
// carried ensemble the exchange index, counter and seed.
void launch_carry(const DevPtrs& d, const DevPtrs& o, int tile, const int2* src, RepState* X, const RepState* Xo,
                  double* T, double* P, const double* To, const double* Po, int nens, const int* sens,
                  const int* rep_off, const int* rep_off_o, const int* nrep_e, int* index, const int* index_o,
                  long long* step, const long long* step_o, unsigned long long* seed,
                  const unsigned long long* seed_o, bool molecules, cudaStream_t s);

}  // namespace remd
