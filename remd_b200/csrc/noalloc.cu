// noalloc.cu -- remd_force_snapshot_noalloc: the FP32 force snapshot of one
// replica, for callers that cannot allocate device memory.
//
// Some host programs own every byte of device memory themselves: a framework
// whose caching allocator has already partitioned the GPU, a plugin host that
// forbids its plugins to allocate, or a loop that must not stall on
// cudaMalloc/cudaFree (both can synchronise the device).  They can still pass
// in their own input and output buffers, but not give the engine its working
// memory.  This entry point therefore keeps all of its scratch -- the
// per-replica constants, the force records, the cell and neighbour lists (skin
// and per-step), the partial sums -- in one file-scope __device__ array of
// fixed size, which every GPU that loads the library holds until the process
// exits.
//
// Limits: at most kNoAllocMaxMol molecules (2048) and a neighbour capacity of
// at most kNoAllocMaxNbr (1024) per molecule, i.e. rcut + 1 A skin <= ~13.4 A.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/remd_b200.h"
#include "engine_types.cuh"
#include "hostio.h"
#include "kernels.cuh"

namespace remd {
namespace {

constexpr int kNoAllocMaxMol = 2048;
constexpr int kNoAllocMaxNbr = 1024;
constexpr int kNoAllocTile = 64;
static_assert(kNoAllocMaxTiles * kNoAllocTile == kNoAllocMaxMol, "one tile per 64 molecules");
constexpr double kNoAllocSkin = 1.0;

constexpr size_t al(size_t x) { return (x + 255) & ~(size_t)255; }
// scratch layout (byte offsets)
constexpr size_t kOffRc = 0;
constexpr size_t kOffTiles = kOffRc + al(sizeof(RepConst));
constexpr size_t kOffState = kOffTiles + al(sizeof(Tile) * kNoAllocMaxTiles);
constexpr size_t kOffR = kOffState + al(sizeof(RepState));
constexpr size_t kOffQ = kOffR + al(8 * 3 * kNoAllocMaxMol);
constexpr size_t kOffF = kOffQ + al(8 * 4 * kNoAllocMaxMol);
constexpr size_t kOffN = kOffF + al(8 * 3 * kNoAllocMaxMol);
constexpr size_t kOffPack = kOffN + al(8 * 4 * kNoAllocMaxMol);
constexpr size_t kOffRef = kOffPack + al(4 * 20 * kNoAllocMaxMol);
constexpr size_t kOffLb = kOffRef + al(sizeof(int4) * kNoAllocMaxMol);
constexpr size_t kOffNbr = kOffLb + al(8 * 3 * kNoAllocMaxTiles);
constexpr size_t kOffNbt = kOffNbr + al(2 * (size_t)kNoAllocMaxNbr * kNoAllocTile * kNoAllocMaxTiles);
constexpr size_t kOffNtc = kOffNbt + al(2 * (size_t)kNoAllocMaxNbr * kNoAllocTile * kNoAllocMaxTiles);
constexpr size_t kOffCom = kOffNtc + al(4 * kNoAllocMaxMol);
constexpr size_t kOffCnt = kOffCom + al(sizeof(int4) * kNoAllocMaxMol);
constexpr size_t kOffPart = kOffCnt + al(4 * kNoAllocMaxMol);
constexpr size_t kOffErr = kOffPart + al(sizeof(Part2) * (kNoAllocMaxMol / 32));
constexpr size_t kOffGrid = kOffErr + al(16);
constexpr size_t kOffCellStart = kOffGrid + al(sizeof(CellGrid));
constexpr size_t kOffCellMol = kOffCellStart + al(4 * (size_t)(kMaxCells + 1));
constexpr size_t kScratchBytes = kOffCellMol + al(sizeof(int4) * (size_t)kNoAllocMaxMol);

// The scratch itself.  On the host this name is only a stand-in for the
// device array: host code must use the address from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_mu;
void* g_scratch_ptr[64] = {nullptr};

// Once per device, with that device current: the device address of the scratch.
int scratch_for_current_device(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return REMD_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      set_error(std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
      return REMD_ERR_CUDA;
    }
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return REMD_OK;
}

}  // namespace
}  // namespace remd

using namespace remd;

extern "C" remd_status remd_force_snapshot_noalloc(const remd_system_desc* s, const double* d_r,
                                                   const double* d_q, const double* L,
                                                   const double* d_wall, double* d_f, double* d_n,
                                                   double* d_out, void* stream) {
  if (!s || !d_r || !d_q || !L || !d_f || !d_n || !d_out) {
    set_error("remd_force_snapshot_noalloc: null argument");
    return REMD_ERR_INVALID;
  }
  // the kernels read d_wall as {f, U} double pairs (16-byte loads) and the
  // other buffers as doubles
  const auto misaligned = [](const void* p, uintptr_t a) { return ((uintptr_t)p % a) != 0; };
  if (misaligned(d_r, 8) || misaligned(d_q, 8) || misaligned(d_f, 8) || misaligned(d_n, 8) ||
      misaligned(d_out, 8) || (d_wall && misaligned(d_wall, 16))) {
    set_error("remd_force_snapshot_noalloc: d_wall must be 16-byte aligned and the other buffers "
              "8-byte aligned");
    return REMD_ERR_INVALID;
  }
  if (s->nmol < 2 || s->nmol > kNoAllocMaxMol) {
    set_error("remd_force_snapshot_noalloc: nmol must be in [2, 2048] (the size of its fixed scratch)");
    return REMD_ERR_INVALID;
  }
  const int ns = s->nsite;
  int c0 = -1;
  if (ns >= 3 && ns <= 5) {
    for (int k = 0; k < ns; k++)
      if (s->site_charge[k] != 0.0) { c0 = k; break; }
    bool ok = c0 >= 0 && s->site_eps[0] > 0.0 && ((ns == 3 && c0 == 0) || (ns >= 4 && c0 == 1));
    for (int k = 1; k < ns && ok; k++) ok = (s->site_eps[k] == 0.0);
    for (int k = (c0 < 0 ? ns : c0); k < ns && ok; k++) ok = (s->site_charge[k] != 0.0);
    if (!ok) c0 = -1;
  }
  if (c0 < 0 || !(s->rcut > s->rswitch) || s->rswitch <= 0.0 || s->confined < 0 || s->confined > 2 ||
      !(L[0] > 0 && L[1] > 0 && L[2] > 0)) {
    set_error("remd_force_snapshot_noalloc: unsupported molecule type, cutoff or box");
    return REMD_ERR_INVALID;
  }
  if (s->confined > 0 && (!d_wall || s->nfwall < 3 || s->wall_length <= 0.0)) {
    set_error("remd_force_snapshot_noalloc: a confined system needs its wall table (remd_wall_table)");
    return REMD_ERR_INVALID;
  }
  const double rl = s->rcut + kNoAllocSkin;
  int cap = ((int)std::ceil(0.1 * 4.0 / 3.0 * M_PI * rl * rl * rl) + 7) / 8 * 8;
  if (cap > s->nmol - 1) cap = s->nmol - 1;
  if (cap > kNoAllocMaxNbr) {
    set_error("remd_force_snapshot_noalloc: rcut too large for its fixed neighbour capacity (1024)");
    return REMD_ERR_INVALID;
  }
  void* base = nullptr;
  int st = scratch_for_current_device(&base);
  if (st != REMD_OK) return (remd_status)st;
  char* b = static_cast<char*>(base);
  cudaStream_t cs = static_cast<cudaStream_t>(stream);

  // per-replica constants, exactly as a one-replica handle builds them
  RepConst c;
  std::memset(&c, 0, sizeof(c));
  c.nmol = s->nmol;
  c.nsite = ns;
  c.c0 = c0;
  c.confined = s->confined;
  c.tconstant = s->tconstant;
  c.pconstant = s->pconstant;
  c.nfwall = s->nfwall;
  c.rc = s->rcut;
  c.rs = s->rswitch;
  const double rlc = s->rswitch - s->rcut;
  c.coef_sw = 1.0 / (rlc * rlc * rlc * rlc * rlc);
  c.skin = kNoAllocSkin;
  c.nbr_cap = cap;
  c.ntile = (s->nmol + kNoAllocTile - 1) / kNoAllocTile;
  c.warp_off = 0;
  c.nwarp = (s->nmol + 31) / 32;
  c.pack_stride = pack_stride(ns, kF32);
  const double wl = s->wall_length * 1e-10 / unit_length();
  c.wall_dr = (s->confined == 2) ? 0.5 * (wl / (double)s->nfwall) : wl / (double)(s->nfwall > 0 ? s->nfwall : 1);
  c.wall_length_param = s->wall_length;
  double qr[kMaxSites];
  for (int k = 0; k < ns; k++) {
    for (int x = 0; x < 3; x++) c.body[k][x] = s->site_r[k][x] * (1e-10 / unit_length());
    qr[k] = s->site_charge[k] * (elementary_charge() / unit_coulomb());
  }
  for (int k = 0; k < ns; k++)
    for (int l = 0; l < ns; l++) c.qq[k][l] = qr[k] * qr[l];
  for (int k = 0; k < ns; k++)
    c.site_reach = std::fmax(c.site_reach, std::sqrt(c.body[k][0] * c.body[k][0] + c.body[k][1] * c.body[k][1] +
                                                     c.body[k][2] * c.body[k][2]));
  const double sg = 0.5 * (s->site_sigma[0] * (1e-10 / unit_length()) * 2.0);
  c.sgm2 = sg * sg;
  const double eo = s->site_eps[0] * (1e+03 / 6.0221367e+23 / unit_energy());
  c.eps = std::sqrt(eo * eo);
  NoAllocSetup setup;
  std::memset(&setup, 0, sizeof(setup));
  setup.c = c;
  for (int t = 0; t < c.ntile; t++) {
    setup.tiles[t].rep = 0;
    setup.tiles[t].start = t * kNoAllocTile;
    setup.tiles[t].count = (s->nmol - t * kNoAllocTile < kNoAllocTile) ? s->nmol - t * kNoAllocTile : kNoAllocTile;
    setup.tiles[t].pad = 0;
  }
  setup.rs.s = 1.0;
  for (int x = 0; x < 3; x++) setup.rs.L[x] = L[x];

  DevPtrs d{};
  d.N = s->nmol;
  d.ntiles = c.ntile;
  d.nrep = 1;
  d.rc = reinterpret_cast<RepConst*>(b + kOffRc);
  d.tiles = reinterpret_cast<Tile*>(b + kOffTiles);
  d.r = reinterpret_cast<double*>(b + kOffR);
  d.q = reinterpret_cast<double*>(b + kOffQ);
  d.f = reinterpret_cast<double*>(b + kOffF);
  d.n = reinterpret_cast<double*>(b + kOffN);
  d.v = d.p = nullptr;
  d.pack = b + kOffPack;
  d.ref_com = reinterpret_cast<int4*>(b + kOffRef);
  d.Lbuild = reinterpret_cast<double*>(b + kOffLb);
  d.nbr = reinterpret_cast<uint16_t*>(b + kOffNbr);
  d.nbt = reinterpret_cast<uint16_t*>(b + kOffNbt);
  d.nt_cnt = reinterpret_cast<int*>(b + kOffNtc);
  d.com = reinterpret_cast<int4*>(b + kOffCom);
  d.nbr_cnt = reinterpret_cast<int*>(b + kOffCnt);
  d.wall = d_wall;
  d.part1 = nullptr;
  d.part2 = reinterpret_cast<Part2*>(b + kOffPart);
  d.err = reinterpret_cast<int*>(b + kOffErr);
  d.status = reinterpret_cast<int*>(b + kOffErr + 4);
  d.cgrid = reinterpret_cast<CellGrid*>(b + kOffGrid);
  d.cell_start = reinterpret_cast<int*>(b + kOffCellStart);
  d.cell_com = reinterpret_cast<int4*>(b + kOffCellMol);
  d.rep0 = 0;
  d.nrep_l = 1;
  d.bm_win = bitmap_window(s->nmol);
  RepState* X = reinterpret_cast<RepState*>(b + kOffState);

  // every earlier call's contents are overwritten before use: constants, tiles
  // and state by the load kernel (from its parameter), records / lists / counts
  // / partial sums by the kernels after it (the load kernel also marks the lists
  // invalid, so they are rebuilt)
  launch_noalloc_load(d, setup, X, d_r, d_q, kNoAllocTile, cs);
  launch_force(d, X, X, kF32, true, kNoAllocTile, cs);
  launch_noalloc_store(d, d_f, d_n, d_out, cs);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string("remd_force_snapshot_noalloc: ") + cudaGetErrorString(e));
    return REMD_ERR_CUDA;
  }
  return REMD_OK;
}
