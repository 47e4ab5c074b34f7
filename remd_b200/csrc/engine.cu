// engine.cu -- host side of the B200 REMD engine: validation, device layout,
// the CUDA-graph interval, and the C-ABI entry points of include/remd_b200.h
// that replace class REMDGPU (src/remdgpu.h:92-238).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <deque>
#include <fstream>
#include <iomanip>
#include <map>
#include <new>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/remd_b200.h"
#include "engine_types.cuh"
#include "hostio.h"
#include "integrator.cuh"
#include "kernels.cuh"

using namespace remd;

#define CK(call)                                                                   \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess) {                                                       \
      set_error(std::string(#call) + ": " + cudaGetErrorString(e_));               \
      return REMD_ERR_CUDA;                                                        \
    }                                                                              \
  } while (0)

constexpr int kMaxChains = 4;   // independent chains of the interval graph

struct remd_engine_s {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t stream2[kMaxChains - 1] = {};   // further chains of the interval graph
  cudaEvent_t ev_fork = nullptr, ev_join[kMaxChains - 1] = {};
  int prec = kF32;
  int tile = 128;
  double skin = 1.0;
  int nens = 0, nrep = 0, N = 0, interval = 0;
  std::vector<remd_system_desc> sys;
  std::vector<int> rep_ens, ens_rep_off, ens_nrep;
  std::vector<RepConst> rc;
  std::vector<Tile> tiles;
  std::vector<int> order;          // force blocks -> tiles, costliest first
  std::vector<int> order2;         // the same per chain: chain k's tiles [chain_tile[k], chain_tile[k+1])
  int nchain = 1;                  // independent chains of the interval graph
  int chain_tile[kMaxChains + 1] = {};
  int chain_rep[kMaxChains + 1] = {};   // chain k's replicas [chain_rep[k], chain_rep[k+1])
  int* d_order2 = nullptr;
  std::vector<double> curT, curP;
  std::vector<double> wall_h;
  DevPtrs d{};
  RepState *X = nullptr, *Y = nullptr;
  void* pool = nullptr;           // one device allocation holds every array
  size_t pool_bytes = 0;
  double *hT = nullptr, *hP = nullptr, *havg = nullptr;   // pinned
  double *dT = nullptr, *dP = nullptr;                    // device conditions
  int* d_index = nullptr;                                 // device exchange index (per replica slot)
  int *d_grid = nullptr, *d_rep_off = nullptr, *d_u_off = nullptr;
  double* d_u = nullptr;
  int u_cap = 0;
  cudaGraphExec_t gexec = nullptr;
  int graph_tile = 0;
  bool graph_exchange = false;
  bool exch_enabled = false;        // device exchange appended to every interval
  bool vscale = false;              // some replica uses velocity scaling (tconstant 2)
  unsigned long long exch_seed = 0;
  long long* d_step = nullptr;      // per-ensemble interval counter of the device exchange
  unsigned long long* d_seed = nullptr;   // per-ensemble Philox seed
  long long last_pairs = 0;
  long long steps_done = 0;        // MD steps run (the simulated time of the .chk Property line)
  double last_graph_ms = 0.0;       // host time of the last interval-graph capture + update/instantiate
  cudaMemPool_t mempool = nullptr;  // the pool comes from this memory pool (serving loop), else cudaMalloc
  int pinned_cap = 0;               // replicas the pinned host buffers hold
  int2* d_carry_src = nullptr;      // per replica: {old first molecule, old replica} of a carried replica
  int* d_carry_ens = nullptr;       // per ensemble: old ensemble or -1
  int* d_ens_nrep = nullptr;        // per ensemble: replicas
  size_t bytes = 0;
  // (volume, potential) histograms per condition slot, per ensemble (own allocations)
  std::vector<HistEns> hist;        // host copy of d_hist (device pointers inside)
  HistEns* d_hist = nullptr;
  int* d_hidx = nullptr;            // slot -> replica index of the last host increment
  std::vector<int> h_hidx;
  bool hist_on = false;             // some ensemble keeps a histogram
  bool graph_hist = false;
};

// Wall tables by their parameters.  The tube table integrates over the wall
// once per entry (about a second of host time for 65536 entries), and a
// serving batch is rebuilt whenever a job joins or leaves it; the tables of the
// jobs still running come from here instead of being computed again.  The
// cache keeps the most recent tables up to kWallCacheBytes in all (1 MB per
// table at 65536 entries), and always the newest one.
using WallKey = std::tuple<int, int, double, double, double, double>;
static WallKey wall_key(const remd_system_desc& s) {
  return WallKey(s.confined, s.nfwall, s.wall_length, s.sgm_wall, s.eps_wall, s.rho_wall);
}
constexpr int kMaxWallEntries = 1 << 24;             // 256 MB per table
constexpr size_t kWallCacheBytes = size_t(256) << 20;
static std::mutex g_wall_mu;
static std::map<WallKey, std::shared_ptr<const std::vector<double>>> g_wall_cache;
static std::deque<WallKey> g_wall_order;   // oldest first
static size_t g_wall_bytes = 0;

static std::shared_ptr<const std::vector<double>> wall_table_cached(const remd_system_desc& s) {
  const WallKey k = wall_key(s);
  {
    std::lock_guard<std::mutex> g(g_wall_mu);
    auto it = g_wall_cache.find(k);
    if (it != g_wall_cache.end()) return it->second;
  }
  auto t = std::make_shared<std::vector<double>>(2 * (size_t)s.nfwall);
  wall_table(s.confined, s.nfwall, s.wall_length, s.sgm_wall, s.eps_wall, s.rho_wall, t->data());
  std::lock_guard<std::mutex> g(g_wall_mu);
  if (g_wall_cache.emplace(k, t).second) {
    g_wall_order.push_back(k);
    g_wall_bytes += t->size() * sizeof(double);
    while (g_wall_bytes > kWallCacheBytes && g_wall_order.size() > 1) {
      auto it = g_wall_cache.find(g_wall_order.front());
      g_wall_bytes -= it->second->size() * sizeof(double);
      g_wall_cache.erase(it);
      g_wall_order.pop_front();
    }
  }
  return t;
}

static int valid_model(const remd_system_desc& s, int* c0) {
  const int ns = s.nsite;
  if (ns < 3 || ns > 5) return 0;
  for (int k = 1; k < ns; k++)
    if (s.site_eps[k] != 0.0) return 0;   // only site 0 is a Lennard-Jones site
  if (s.site_eps[0] <= 0.0) return 0;
  int first = -1;
  for (int k = 0; k < ns; k++)
    if (s.site_charge[k] != 0.0) { first = k; break; }
  if (first < 0) return 0;
  for (int k = first; k < ns; k++)
    if (s.site_charge[k] == 0.0) return 0;
  if (!((ns == 3 && first == 0) || (ns >= 4 && first == 1))) return 0;
  *c0 = first;
  return 1;
}

static remd_status check_desc(const remd_system_desc& s, std::string& why) {
  int c0;
  if (s.nmol < 2 || s.nmol > 65535) { why = "nmol must be in [2, 65535]"; return REMD_ERR_INVALID; }
  if (!valid_model(s, &c0)) {
    why = "molecule type: site 0 must be the only LJ site and the charged sites a contiguous tail "
          "(TIP3P/TIP4P/TIP5P layout)";
    return REMD_ERR_INVALID;
  }
  if (s.tconstant < 0 || s.tconstant > 2) { why = "tconstant must be 0, 1 or 2"; return REMD_ERR_INVALID; }
  // velocity scaling: the modes Molecules::ExecuteSteps integrates (src/integrator.cxx:730-787:
  // NVTSCALE, NVTSCALE1D, NAxyPzTSCALE1D); the other *TSCALE* modes fall through its switch
  // and are not integrated at all there, so they are rejected here
  if (s.tconstant == 2 && !((s.confined == 0 && s.pconstant == 0) ||
                            (s.confined == 1 && (s.pconstant == 0 || s.pconstant == 2)))) {
    why = "tconstant 2 (velocity scaling) is integrated for bulk pconstant 0 and tube pconstant 0 or 2 only";
    return REMD_ERR_INVALID;
  }
  if (s.pconstant < 0 || s.pconstant > 3) { why = "pconstant must be 0..3"; return REMD_ERR_INVALID; }
  if (s.confined < 0 || s.confined > 2) { why = "confined must be 0..2"; return REMD_ERR_INVALID; }
  // src/remd.cxx:35-36
  if (s.confined == 1 && (s.pconstant == 1 || s.pconstant == 3)) { why = "tube needs pconstant 0 or 2"; return REMD_ERR_INVALID; }
  if (s.confined == 2 && (s.pconstant == 1 || s.pconstant == 2)) { why = "slit needs pconstant 0 or 3"; return REMD_ERR_INVALID; }
  if (s.confined > 0 && (s.nfwall < 3 || s.wall_length <= 0.0)) { why = "confined system needs nfwall >= 3 and wall_length > 0"; return REMD_ERR_INVALID; }
  if (s.confined > 0 && s.nfwall > kMaxWallEntries) { why = "nfwall must be <= 16777216"; return REMD_ERR_INVALID; }
  if (!(s.rcut > s.rswitch) || s.rswitch <= 0.0) { why = "need rcut > rswitch > 0"; return REMD_ERR_INVALID; }
  if (s.interval < 1) { why = "interval must be >= 1"; return REMD_ERR_INVALID; }
  if (!(s.dt_fs > 0.0)) { why = "dt must be > 0"; return REMD_ERR_INVALID; }
  return REMD_OK;
}

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Build RepConst/tiles for the current tile size; returns pool layout size.
static void layout(remd_engine_s* h, std::vector<size_t>& offs, size_t& total) {
  const int T = h->tile;
  h->tiles.clear();
  long long pack_words = 0, nbr_words = 0;
  int nwarps = 0;
  for (int r = 0; r < h->nrep; r++) {
    RepConst& c = h->rc[r];
    c.tile_off = (int)h->tiles.size();
    c.ntile = (c.nmol + T - 1) / T;
    c.warp_off = nwarps;
    c.nwarp = (c.nmol + 31) / 32;
    nwarps += c.nwarp;
    for (int t = 0; t < c.ntile; t++) {
      Tile tt;
      tt.rep = r;
      tt.start = t * T;
      tt.count = std::min(T, c.nmol - t * T);
      tt.pad = 0;
      h->tiles.push_back(tt);
    }
    c.pack_stride = pack_stride(c.nsite, h->prec);
    c.pack_off = pack_words;
    pack_words += (long long)c.nmol * c.pack_stride;
    c.nbr_off = nbr_words;
    nbr_words += (long long)c.ntile * c.nbr_cap * T;
  }
  // force blocks in decreasing order of estimated pair work (longest first, so
  // the costliest tiles do not form the tail of the launch): molecules x
  // neighbours within rcut at liquid density x FLOPs per molecule pair
  {
    std::vector<double> cost(h->tiles.size());
    for (size_t t = 0; t < h->tiles.size(); t++) {
      const RepConst& c = h->rc[h->tiles[t].rep];
      const double nbr = std::min((double)(c.nmol - 1), 0.0334 * 4.0 / 3.0 * M_PI * c.rc * c.rc * c.rc);
      const int nq = c.nsite - c.c0;
      cost[t] = h->tiles[t].count * nbr * (51.0 + 32.0 + 27.0 * nq * nq);
    }
    h->order.resize(h->tiles.size());
    for (size_t t = 0; t < h->order.size(); t++) h->order[t] = (int)t;
    std::stable_sort(h->order.begin(), h->order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    // groups of whole replicas of about equal cost (boundaries at the replica
    // boundaries nearest k/K of the total) for the independent chains of the
    // interval graph
    const int K = std::min(kMaxChains, h->nrep);
    std::vector<double> before(h->nrep + 1, 0.0);   // cost of replicas [0, r)
    for (int r = 0; r < h->nrep; r++) {
      double w = 0.0;
      for (int t = h->rc[r].tile_off; t < h->rc[r].tile_off + h->rc[r].ntile; t++) w += cost[t];
      before[r + 1] = before[r] + w;
    }
    std::vector<int> cut(1, 0);   // first replica of each chain
    for (int k = 1; k < K; k++) {
      const double goal = before[h->nrep] * k / K;
      int best = cut.back() + 1;
      for (int r = cut.back() + 1; r <= h->nrep - (K - k); r++)
        if (std::fabs(before[r] - goal) < std::fabs(before[best] - goal)) best = r;
      cut.push_back(best);
    }
    h->nchain = K;
    for (int k = 0; k < K; k++) {
      h->chain_tile[k] = h->rc[cut[k]].tile_off;
      h->chain_rep[k] = cut[k];
    }
    h->chain_tile[K] = (int)h->tiles.size();
    h->chain_rep[K] = h->nrep;
    h->order2.clear();
    for (int k = 0; k < K; k++)
      for (int t : h->order)
        if (t >= h->chain_tile[k] && t < h->chain_tile[k + 1]) h->order2.push_back(t);
  }
  const size_t N = h->N, nt = h->tiles.size(), nr = h->nrep;
  const size_t elem = (h->prec == kF32) ? 4 : 8;
  const size_t sizes[] = {
      nr * sizeof(RepConst),           // 0 rc
      nt * sizeof(Tile),               // 1 tiles
      N * 3 * 8, N * 3 * 8, N * 4 * 8, N * 4 * 8, N * 3 * 8, N * 4 * 8,   // 2..7 r v q p f n
      (size_t)pack_words * elem,       // 8 pack
      N * sizeof(int4),                // 9 ref_com
      nt * 3 * 8,                      // 10 Lbuild
      (size_t)nbr_words * 2,           // 11 nbr
      N * 4,                           // 12 nbr_cnt
      std::max<size_t>(h->wall_h.size(), 2) * 8,   // 13 wall
      (size_t)nwarps * sizeof(Part1), (size_t)nwarps * sizeof(Part2),   // 14, 15 (per 32 molecules)
      nr * kNumAvg * 8,                // 16 avg
      nr * 4, 64,                      // 17 status, 18 err
      nr * 8, nr * 8,                  // 19 T, 20 P
      nr * sizeof(RepState), nr * sizeof(RepState),   // 21 X, 22 Y
      nr * 4,                          // 23 index
      (size_t)h->nens * 2 * 4, (size_t)h->nens * 4, (size_t)h->nens * 4,   // 24 grid 25 rep_off 26 u_off
      (size_t)std::max(nr / 2, (size_t)1) * 8,   // 27 u
      (size_t)h->nens * 8,             // 28 per-ensemble exchange step counter
      (size_t)h->nens * 8,             // 29 per-ensemble exchange seed
      (h->prec == kF32) ? (size_t)nbr_words * 2 : 0,   // 30 nbt (FP32 per-step lists)
      nt * 4,                          // 31 order
      (h->prec == kF32) ? N * 4 : 0,   // 32 nt_cnt (FP32 per-step list counts)
      N * sizeof(int4),                // 33 com (FP32 current fixed-point centres)
      nt * 4,                          // 34 order per chain (multi-chain interval graph)
      nr * sizeof(CellGrid),           // 35 cell grid + rebuild decision per replica
      nr * (size_t)(kMaxCells + 1) * 4,   // 36 cell offsets per replica
      N * sizeof(int4),                // 37 centres sorted by cell
      nr * sizeof(int2),               // 38 carried replicas' sources (serving batch changes)
      (size_t)h->nens * 4, (size_t)h->nens * 4,   // 39 carried ensembles' sources, 40 replicas per ensemble
  };
  offs.clear();
  total = 0;
  for (size_t s : sizes) {
    offs.push_back(total);
    total += align256(s);
  }
}

static void free_pool(remd_engine_s* h) {
  if (h->mempool) cudaFreeAsync(h->pool, h->stream);
  else cudaFree(h->pool);
  h->pool = nullptr;
}

static remd_status allocate(remd_engine_s* h) {
  std::vector<size_t> offs;
  size_t total;
  layout(h, offs, total);
  if (h->pool) { free_pool(h); }
  cudaError_t e = h->mempool ? cudaMallocFromPoolAsync(&h->pool, total, h->mempool, h->stream)
                             : cudaMalloc(&h->pool, total);
  if (e != cudaSuccess) {
    set_error(std::string("device allocation of ") + std::to_string(total) + " bytes: " + cudaGetErrorString(e));
    return REMD_ERR_OOM;
  }
  h->pool_bytes = total;
  char* b = static_cast<char*>(h->pool);
  CK(cudaMemsetAsync(b, 0, total, h->stream));
  DevPtrs& d = h->d;
  d.N = h->N;
  d.ntiles = (int)h->tiles.size();
  d.nrep = h->nrep;
  d.rc = reinterpret_cast<RepConst*>(b + offs[0]);
  d.tiles = reinterpret_cast<Tile*>(b + offs[1]);
  d.r = reinterpret_cast<double*>(b + offs[2]);
  d.v = reinterpret_cast<double*>(b + offs[3]);
  d.q = reinterpret_cast<double*>(b + offs[4]);
  d.p = reinterpret_cast<double*>(b + offs[5]);
  d.f = reinterpret_cast<double*>(b + offs[6]);
  d.n = reinterpret_cast<double*>(b + offs[7]);
  d.pack = b + offs[8];
  d.ref_com = reinterpret_cast<int4*>(b + offs[9]);
  d.Lbuild = reinterpret_cast<double*>(b + offs[10]);
  d.nbr = reinterpret_cast<uint16_t*>(b + offs[11]);
  d.nbr_cnt = reinterpret_cast<int*>(b + offs[12]);
  d.wall = reinterpret_cast<double*>(b + offs[13]);
  d.part1 = reinterpret_cast<Part1*>(b + offs[14]);
  d.part2 = reinterpret_cast<Part2*>(b + offs[15]);
  d.avg = reinterpret_cast<double*>(b + offs[16]);
  d.status = reinterpret_cast<int*>(b + offs[17]);
  d.err = reinterpret_cast<int*>(b + offs[18]);
  h->dT = reinterpret_cast<double*>(b + offs[19]);
  h->dP = reinterpret_cast<double*>(b + offs[20]);
  d.newT = h->dT;
  d.newP = h->dP;
  d.changed = nullptr;
  h->X = reinterpret_cast<RepState*>(b + offs[21]);
  h->Y = reinterpret_cast<RepState*>(b + offs[22]);
  h->d_index = reinterpret_cast<int*>(b + offs[23]);
  h->d_grid = reinterpret_cast<int*>(b + offs[24]);
  h->d_rep_off = reinterpret_cast<int*>(b + offs[25]);
  h->d_u_off = reinterpret_cast<int*>(b + offs[26]);
  h->d_u = reinterpret_cast<double*>(b + offs[27]);
  h->d_step = reinterpret_cast<long long*>(b + offs[28]);
  h->d_seed = reinterpret_cast<unsigned long long*>(b + offs[29]);
  d.nbt = reinterpret_cast<uint16_t*>(b + offs[30]);
  d.order = reinterpret_cast<int*>(b + offs[31]);
  d.nt_cnt = reinterpret_cast<int*>(b + offs[32]);
  d.com = reinterpret_cast<int4*>(b + offs[33]);
  d.tile0 = 0;
  h->d_order2 = reinterpret_cast<int*>(b + offs[34]);
  d.cgrid = reinterpret_cast<CellGrid*>(b + offs[35]);
  d.cell_start = reinterpret_cast<int*>(b + offs[36]);
  d.cell_com = reinterpret_cast<int4*>(b + offs[37]);
  h->d_carry_src = reinterpret_cast<int2*>(b + offs[38]);
  h->d_carry_ens = reinterpret_cast<int*>(b + offs[39]);
  h->d_ens_nrep = reinterpret_cast<int*>(b + offs[40]);
  d.rep0 = 0;
  d.nrep_l = h->nrep;
  {
    int nmax = 1;
    for (const RepConst& c : h->rc) nmax = std::max(nmax, c.nmol);
    d.bm_win = bitmap_window(nmax);
  }
  h->u_cap = std::max(h->nrep / 2, 1);
  h->bytes = total;
  CK(cudaMemcpyAsync((void*)d.rc, h->rc.data(), h->rc.size() * sizeof(RepConst), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync((void*)d.tiles, h->tiles.data(), h->tiles.size() * sizeof(Tile), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync((void*)d.order, h->order.data(), h->order.size() * sizeof(int), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_order2, h->order2.data(), h->order2.size() * sizeof(int), cudaMemcpyHostToDevice, h->stream));
  if (!h->wall_h.empty())
    CK(cudaMemcpyAsync((void*)d.wall, h->wall_h.data(), h->wall_h.size() * 8, cudaMemcpyHostToDevice, h->stream));
  // later set-up copies use the default stream, which does not order with this
  // non-blocking stream: finish the clear and the uploads first
  CK(cudaStreamSynchronize(h->stream));
  return REMD_OK;
}

// Waits for the handle's stream and reports the device error word.  The word
// is cleared once read, so an error is reported by the call whose work raised
// it and a later call starts clean (a replica that stays non-finite raises it
// again; its per-replica status word keeps the cause).
static remd_status sync_and_check(remd_engine_s* h) {
  CK(cudaStreamSynchronize(h->stream));
  int err = 0;
  CK(cudaMemcpy(&err, h->d.err, sizeof(int), cudaMemcpyDeviceToHost));
  if (err != 0) CK(cudaMemset(h->d.err, 0, sizeof(int)));
  if (err & kErrNbrOverflow) {
    set_error("neighbour list capacity exceeded");
    return REMD_ERR_NEIGHBOR_OVERFLOW;
  }
  if (err & kErrNonFinite) {
    set_error("a replica produced a non-finite energy (see remd_replica_status)");
    return REMD_ERR_NONFINITE;
  }
  if (err & kErrHistRange) {
    set_error("potential energy or volume is not in the histogram range");
    return REMD_ERR_RANGE;
  }
  return REMD_OK;
}

// Upload SoA state from host copies (component-major).
static remd_status upload_state(remd_engine_s* h, const std::vector<double>& r, const std::vector<double>& v,
                                const std::vector<double>& q, const std::vector<double>& p,
                                const std::vector<RepState>& st) {
  const size_t N = h->N;
  CK(cudaMemcpyAsync(h->d.r, r.data(), N * 3 * 8, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d.v, v.data(), N * 3 * 8, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d.q, q.data(), N * 4 * 8, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d.p, p.data(), N * 4 * 8, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->X, st.data(), st.size() * sizeof(RepState), cudaMemcpyHostToDevice, h->stream));
  return REMD_OK;
}

static remd_status initial_force(remd_engine_s* h) {
  launch_pack(h->d, h->prec, h->tile, h->stream);
  launch_force(h->d, h->X, h->X, h->prec, true, h->tile, h->stream);
  launch_replica_props(h->d, h->X, h->stream);
  CK(cudaGetLastError());
  return sync_and_check(h);
}

// The integrate part of MD step s of an interval.  With velocity-scaling
// replicas (tconstant 2) every step first closes the previous one
// (k_replica_end: the last half kick), rescales the velocities of those replicas
// (VelocityScaling + AngVelocityScaling before every step, as
// Molecules::ExecuteSteps does, src/integrator.cxx:713-723) and opens the step;
// the other replicas' arithmetic is the same as in the fused closing + opening.
static void launch_step_integrate(remd_engine_s* h, int s) {
  if (h->vscale) {
    if (s > 0) launch_replica_end(h->d, h->X, h->stream);
    launch_replica_rescale(h->d, h->X, true, h->stream);
    launch_integrate_prec(h->d, h->X, h->Y, false, h->tile, h->prec, h->stream);
  } else {
    launch_integrate_prec(h->d, h->X, h->Y, s > 0, h->tile, h->prec, h->stream);
  }
}

static remd_status build_graph(remd_engine_s* h) {
  cudaGraph_t g;
  CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  launch_replica_start(h->d, h->X, h->stream);
  if (h->nchain > 1 && !h->vscale) {
    // independent chains, one per group of replicas (no data crosses between
    // them), so one group's latency-bound phases -- the integrate kernel's
    // scalar chains, the list kernel's heads, the pair kernel's tail -- overlap
    // the other groups' work
    DevPtrs dg[kMaxChains];
    for (int k = 0; k < h->nchain; k++) {
      dg[k] = h->d;
      dg[k].ntiles = h->chain_tile[k + 1] - h->chain_tile[k];
      dg[k].order = h->d_order2 + h->chain_tile[k];
      dg[k].tile0 = h->chain_tile[k];
      dg[k].rep0 = h->chain_rep[k];
      dg[k].nrep_l = h->chain_rep[k + 1] - h->chain_rep[k];
    }
    cudaEventRecord(h->ev_fork, h->stream);
    for (int k = 1; k < h->nchain; k++) cudaStreamWaitEvent(h->stream2[k - 1], h->ev_fork, 0);
    for (int s = 0; s < h->interval; s++)
      for (int k = 0; k < h->nchain; k++) {
        cudaStream_t st = k ? h->stream2[k - 1] : h->stream;
        launch_integrate_prec(dg[k], h->X, h->Y, s > 0, h->tile, h->prec, st);
        launch_force(dg[k], h->Y, h->X, h->prec, false, h->tile, st);
      }
    for (int k = 1; k < h->nchain; k++) {
      cudaEventRecord(h->ev_join[k - 1], h->stream2[k - 1]);
      cudaStreamWaitEvent(h->stream, h->ev_join[k - 1], 0);
    }
  } else {
    for (int s = 0; s < h->interval; s++) {
      launch_step_integrate(h, s);
      launch_force(h->d, h->Y, h->X, h->prec, false, h->tile, h->stream);
    }
  }
  launch_replica_end(h->d, h->X, h->stream);
  // the histogram samples the interval before the exchange moves the conditions
  // (REMD::ExecuteREMD: IncrementHistogram, then ReplicaExchange, src/remd.cxx:396-401)
  if (h->exch_enabled && h->hist_on)
    launch_histogram(h->d, h->d_hist, h->d_rep_off, h->d_index, h->stream);
  if (h->exch_enabled)
    launch_exchange_k(h->d, h->d_grid, h->d_rep_off, h->d_u_off, h->nens, -1, nullptr, h->d_seed,
                      h->d_index, h->dT, h->dP, h->d_step, h->stream);
  cudaError_t le = cudaGetLastError();
  cudaError_t ce = cudaStreamEndCapture(h->stream, &g);
  if (le != cudaSuccess || ce != cudaSuccess) {
    set_error(std::string("graph capture: ") + cudaGetErrorString(le != cudaSuccess ? le : ce));
    return REMD_ERR_CUDA;
  }
  // an existing executable graph of the same topology (the handle's previous
  // graph, or the one a carried handle took over) is updated in place, which
  // costs far less than instantiating a new one
  if (h->gexec) {
    cudaGraphExecUpdateResultInfo info;
    if (cudaGraphExecUpdate(h->gexec, g, &info) == cudaSuccess) {
      cudaGraphDestroy(g);
      h->graph_tile = h->tile;
      h->graph_exchange = h->exch_enabled;
      h->graph_hist = h->hist_on;
      return REMD_OK;
    }
    cudaGetLastError();
    cudaGraphExecDestroy(h->gexec);
    h->gexec = nullptr;
  }
  cudaError_t ie = cudaGraphInstantiate(&h->gexec, g, 0);
  cudaGraphDestroy(g);
  if (ie != cudaSuccess) {
    set_error(std::string("graph instantiate: ") + cudaGetErrorString(ie));
    return REMD_ERR_CUDA;
  }
  h->graph_tile = h->tile;
  h->graph_exchange = h->exch_enabled;
  h->graph_hist = h->hist_on;
  return REMD_OK;
}

static long long host_pairs(remd_engine_s* h) {
  const RepConst& last = h->rc.back();
  std::vector<Part2> p2((size_t)last.warp_off + last.nwarp);
  if (cudaMemcpy(p2.data(), h->d.part2, p2.size() * sizeof(Part2), cudaMemcpyDeviceToHost) != cudaSuccess)
    return -1;
  long long s = 0;
  for (auto& p : p2) s += p.npairs;
  return s / 2;
}

namespace remd {

remd_status engine_get_exchange(remd_handle h, long long* steps, int* index) {
  CK(cudaStreamSynchronize(h->stream));
  CK(cudaMemcpy(steps, h->d_step, h->nens * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(index, h->d_index, h->nrep * 4, cudaMemcpyDeviceToHost));
  return REMD_OK;
}

size_t engine_bytes(remd_handle h) { return h ? h->bytes : 0; }

void engine_prepare_wall(const remd_system_desc& s) {
  std::string why;
  try {
    if (s.confined > 0 && check_desc(s, why) == REMD_OK) wall_table_cached(s);
  } catch (...) {
    // out of host memory: the job's handle build computes the table again and reports it
  }
}

double engine_last_graph_ms(remd_handle h) { return h ? h->last_graph_ms : 0.0; }

remd_status engine_create_carry(remd_handle from, const remd_system_desc* systems, int nens,
                                const int* reps_per_ens, const remd_replica_init* reps, const int* src_rep,
                                const int* src_ens, const int* grids, const unsigned long long* seeds,
                                const long long* steps, remd_precision prec, int device, cudaMemPool_t mempool,
                                remd_handle* out);

}  // namespace remd

// A new handle that continues replicas of an existing one (the serving loop's
// batch changes): their molecule state, scalars, pending condition and, per
// ensemble, the exchange's index, counter and seed are copied on the device
// from `from`, which must be on the same device with the same precision; the
// new handle takes over its streams, pinned buffers and interval graph (updated
// in place at the first interval when its topology allows).  `reps` entries of
// carried replicas are not read.
struct Carry {
  remd_engine_s* from;
  const int* src_rep;                // per new replica: its replica in `from`, or -1
  const int* src_ens;                // per new ensemble: its ensemble in `from`, or -1
  const int* grids;                  // ntemp, npress per ensemble (device exchange)
  const unsigned long long* seeds;   // per ensemble (read for new ensembles)
  const long long* steps;            // per ensemble (read for new ensembles)
  cudaMemPool_t mempool;             // the new pool's memory pool (may be NULL)
};

// The device exchange configuration of a carried handle and the carried
// replicas' state, then the initial force of every replica (forces are a pure
// function of the positions, so a carried replica's are the ones it had), H0 of
// the new replicas (InitializeProperty) and the carried replicas' scalars again
// (their H0 and gkT, which the property pass recomputes).
static remd_status carry_in(remd_engine_s* h, const Carry* cy) {
  remd_engine_s* o = cy->from;
  std::vector<int2> src(h->nrep);
  for (int k = 0; k < h->nrep; k++) {
    const int so = o ? cy->src_rep[k] : -1;
    src[k] = make_int2(so >= 0 ? o->rc[so].mol_off : -1, so);
  }
  std::vector<int> sens(cy->src_ens, cy->src_ens + h->nens);
  if (!o) std::fill(sens.begin(), sens.end(), -1);
  std::vector<int> idx(h->nrep);
  for (int e = 0; e < h->nens; e++)
    for (int k = 0; k < h->ens_nrep[e]; k++) idx[h->ens_rep_off[e] + k] = k;
  CK(cudaMemcpyAsync(h->d_carry_src, src.data(), src.size() * sizeof(int2), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_carry_ens, sens.data(), sens.size() * 4, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_ens_nrep, h->ens_nrep.data(), h->nens * 4, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_grid, cy->grids, 2 * h->nens * 4, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_seed, cy->seeds, h->nens * 8, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_step, cy->steps, h->nens * 8, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_index, idx.data(), idx.size() * 4, cudaMemcpyHostToDevice, h->stream));
  auto carry = [&](bool molecules) {
    if (!o) return;
    launch_carry(h->d, o->d, h->tile, h->d_carry_src, h->X, o->X, h->dT, h->dP, o->dT, o->dP, h->nens,
                 h->d_carry_ens, h->d_rep_off, o->d_rep_off, h->d_ens_nrep, h->d_index, o->d_index, h->d_step,
                 o->d_step, h->d_seed, o->d_seed, molecules, h->stream);
  };
  carry(true);
  launch_pack(h->d, h->prec, h->tile, h->stream);
  launch_force(h->d, h->X, h->X, h->prec, true, h->tile, h->stream);
  launch_replica_props(h->d, h->X, h->stream);
  carry(false);
  CK(cudaGetLastError());
  h->exch_enabled = true;
  // the host copies of the current conditions (read by remd_execute_steps)
  if (o)
    for (int k = 0; k < h->nrep; k++)
      if (cy->src_rep[k] >= 0) { h->curT[k] = o->curT[cy->src_rep[k]]; h->curP[k] = o->curP[cy->src_rep[k]]; }
  return sync_and_check(h);
}

// A carried handle that could not be built gives the previous handle back what
// it took over (streams, events, graph, pinned buffers), then is destroyed: the
// previous batch stays usable.
static void undo_carry(remd_engine_s* h, const Carry* cy) {
  if (cy && cy->from) {
    remd_engine_s* o = cy->from;
    if (h->stream) cudaStreamSynchronize(h->stream);   // nothing of h's is in flight any more
    if (h->pool) free_pool(h);
    if (!o->stream) { o->stream = h->stream; h->stream = nullptr; }
    if (!o->ev_fork) { o->ev_fork = h->ev_fork; h->ev_fork = nullptr; }
    for (int k = 0; k < kMaxChains - 1; k++) {
      if (!o->stream2[k]) { o->stream2[k] = h->stream2[k]; h->stream2[k] = nullptr; }
      if (!o->ev_join[k]) { o->ev_join[k] = h->ev_join[k]; h->ev_join[k] = nullptr; }
    }
    if (!o->gexec) { o->gexec = h->gexec; h->gexec = nullptr; }
    if (!o->hT) {
      o->hT = h->hT; o->hP = h->hP; o->havg = h->havg; o->pinned_cap = h->pinned_cap;
      h->hT = h->hP = h->havg = nullptr;
    }
  }
  remd_destroy(h);
}

static remd_status create_impl(const remd_system_desc* systems, int nens, const int* reps_per_ens,
                               const remd_replica_init* reps, remd_precision prec, int device,
                               const Carry* cy, remd_handle* out) {
  if (!systems || nens < 1 || !reps_per_ens || !reps || !out) {
    set_error("remd_create: null argument");
    return REMD_ERR_INVALID;
  }
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
    set_error("no CUDA device");
    return REMD_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= ndev) { set_error("bad device"); return REMD_ERR_INVALID; }
  std::string why;
  for (int e = 0; e < nens; e++) {
    remd_status st = check_desc(systems[e], why);
    if (st != REMD_OK) { set_error("system " + std::to_string(e) + ": " + why); return st; }
    if (systems[e].interval != systems[0].interval) {
      set_error("all systems of one handle must share `interval`");
      return REMD_ERR_INVALID;
    }
    if (reps_per_ens[e] < 1) { set_error("reps_per_ens must be >= 1"); return REMD_ERR_INVALID; }
  }
  auto* h = new remd_engine_s;
  h->device = device;
  h->prec = (prec == REMD_PREC_FP64) ? kF64 : kF32;
  h->tile = (h->prec == kF32) ? 32 : 128;   // measured best on a 256-replica mixed batch; remd_set_tuning / remd_autotune change it
  h->nens = nens;
  h->interval = systems[0].interval;
  h->sys.assign(systems, systems + nens);
  // wall tables: one per distinct set of wall parameters, shared by the
  // ensembles that have it
  std::vector<int> wall_off(nens, 0);
  for (int e = 0; e < nens; e++) {
    const remd_system_desc& s = systems[e];
    if (s.confined <= 0) continue;
    int same = -1;
    for (int f = 0; f < e && same < 0; f++)
      if (wall_key(systems[f]) == wall_key(s)) same = f;
    if (same >= 0) { wall_off[e] = wall_off[same]; continue; }
    if (h->wall_h.size() / 2 + (size_t)s.nfwall > (size_t)INT32_MAX) {
      set_error("system " + std::to_string(e) + ": the handle's wall tables exceed 2^31 entries");
      delete h;
      return REMD_ERR_INVALID;
    }
    wall_off[e] = (int)(h->wall_h.size() / 2);
    try {
      const auto t = wall_table_cached(s);
      h->wall_h.insert(h->wall_h.end(), t->begin(), t->end());
    } catch (const std::bad_alloc&) {
      set_error("system " + std::to_string(e) + ": no host memory for the wall table");
      delete h;
      return REMD_ERR_OOM;
    }
  }
  // replicas
  int rep = 0, mol = 0;
  std::vector<RepState> st0;
  for (int e = 0; e < nens; e++) {
    const remd_system_desc& s = systems[e];
    h->ens_rep_off.push_back(rep);
    h->ens_nrep.push_back(reps_per_ens[e]);
    int c0 = 0;
    valid_model(s, &c0);
    for (int k = 0; k < reps_per_ens[e]; k++, rep++) {
      const int src = (cy && cy->from) ? cy->src_rep[rep] : -1;
      remd_replica_init ri = reps[rep];
      std::vector<double> cm, ci;   // a carried replica's mass and inertia columns
      if (src >= 0) {
        const RepConst& o = cy->from->rc[src];
        cm.assign(s.nmol, o.mass);
        ci.resize(3 * (size_t)s.nmol);
        for (int i = 0; i < s.nmol; i++)
          for (int x = 0; x < 3; x++) ci[3 * i + x] = o.I[x];
        ri.r = ri.v = ri.q = ri.p = cm.data();   // not read: the state is copied on the device
        ri.mass = cm.data();
        ri.inertia = ci.data();
        ri.Q = o.Q;
        ri.W = o.W;
        ri.T = cy->from->curT[src];
        ri.P = cy->from->curP[src];
        ri.s = 1.0;
        ri.Ps = 0.0;
        for (int x = 0; x < 3; x++) { ri.Pv[x] = 0.0; ri.L[x] = 1.0; }   // replaced on the device
      }
      if (!ri.r || !ri.v || !ri.q || !ri.p || !ri.mass || !ri.inertia) {
        set_error("replica " + std::to_string(rep) + ": null state array");
        delete h;
        return REMD_ERR_INVALID;
      }
      for (int i = 1; i < s.nmol; i++) {
        if (ri.mass[i] != ri.mass[0] || ri.inertia[3 * i] != ri.inertia[0] ||
            ri.inertia[3 * i + 1] != ri.inertia[1] || ri.inertia[3 * i + 2] != ri.inertia[2]) {
          set_error("replica " + std::to_string(rep) + ": molecules of one replica must share mass and inertia");
          delete h;
          return REMD_ERR_INVALID;
        }
      }
      if (!(ri.Q > 0.0) || (s.pconstant > 0 && !(ri.W > 0.0)) || !(ri.T > 0.0) ||
          !(ri.L[0] > 0 && ri.L[1] > 0 && ri.L[2] > 0) || !(ri.s > 0.0)) {
        set_error("replica " + std::to_string(rep) + ": need Q > 0, W > 0 (barostat), T > 0, L > 0, s > 0");
        delete h;
        return REMD_ERR_INVALID;
      }
      RepConst c;
      std::memset(&c, 0, sizeof(c));
      c.nmol = s.nmol;
      c.mol_off = mol;
      c.nsite = s.nsite;
      c.c0 = c0;
      c.confined = s.confined;
      c.tconstant = s.tconstant;
      if (s.tconstant == 2) h->vscale = true;
      c.pconstant = s.pconstant;
      c.nfwall = s.nfwall;
      c.wall_off = wall_off[e];
      c.ens = e;
      c.dt = s.dt_fs * 1e-15 / unit_time();
      c.dthalf = s.dt_fs * 1e-15 / unit_time() * 0.5;
      c.rc = s.rcut;
      c.rs = s.rswitch;
      const double rlc = s.rswitch - s.rcut;
      c.coef_sw = 1.0 / (rlc * rlc * rlc * rlc * rlc);
      c.skin = h->skin;
      c.Q = ri.Q;
      c.W = ri.W > 0.0 ? ri.W : 1.0;
      c.mass = ri.mass[0];
      for (int x = 0; x < 3; x++) c.I[x] = ri.inertia[x];
      const double wl = s.wall_length * 1e-10 / unit_length();
      c.wall_dr = (s.confined == 2) ? 0.5 * (wl / (double)s.nfwall) : wl / (double)std::max(s.nfwall, 1);
      c.wall_length_param = s.wall_length;
      const double sigma_c = 3.4;
      const double wa = (s.wall_length - 0.5 * sigma_c) * 1e-10 / unit_length();
      c.bottom_area = M_PI * wa * wa;
      c.slit_width = s.wall_length * 1e-10 / unit_length();
      double qr[kMaxSites];
      for (int k = 0; k < s.nsite; k++) {
        for (int x = 0; x < 3; x++) c.body[k][x] = s.site_r[k][x] * (1e-10 / unit_length());
        qr[k] = s.site_charge[k] * (elementary_charge() / unit_coulomb());
      }
      for (int k = 0; k < s.nsite; k++)
        for (int l = 0; l < s.nsite; l++) c.qq[k][l] = qr[k] * qr[l];
      c.site_reach = 0.0;
      for (int k = 0; k < s.nsite; k++)
        c.site_reach = std::max(c.site_reach, std::sqrt(c.body[k][0] * c.body[k][0] + c.body[k][1] * c.body[k][1] +
                                                        c.body[k][2] * c.body[k][2]));
      const double sg = 0.5 * (s.site_sigma[0] * (1e-10 / unit_length()) * 2.0);
      c.sgm2 = sg * sg;
      const double eo = s.site_eps[0] * (1e+03 / 6.0221367e+23 / unit_energy());
      c.eps = std::sqrt(eo * eo);
      const double rl = s.rcut + h->skin;
      const double cap = 0.1 * 4.0 / 3.0 * M_PI * rl * rl * rl;
      c.nbr_cap = std::min(s.nmol - 1, ((int)std::ceil(cap) + 7) / 8 * 8);
      if (c.nbr_cap < 1) c.nbr_cap = 1;
      h->rc.push_back(c);
      h->rep_ens.push_back(e);
      RepState rs;
      std::memset(&rs, 0, sizeof(rs));
      rs.s = ri.s;
      rs.Ps = ri.Ps;
      for (int x = 0; x < 3; x++) { rs.Pv[x] = ri.Pv[x]; rs.L[x] = ri.L[x]; }
      rs.T = ri.T;
      rs.P = ri.P;
      rs.gkT = 6.0 * s.nmol * ri.T;
      st0.push_back(rs);
      h->curT.push_back(ri.T);
      h->curP.push_back(ri.P);
      mol += s.nmol;
    }
  }
  h->nrep = rep;
  h->N = mol;
  h->mempool = cy ? cy->mempool : nullptr;
  if (cy && cy->from) {
    remd_engine_s* o = cy->from;
    h->stream = o->stream;
    h->ev_fork = o->ev_fork;
    o->stream = nullptr;
    o->ev_fork = nullptr;
    for (int k = 0; k < kMaxChains - 1; k++) {
      h->stream2[k] = o->stream2[k];
      h->ev_join[k] = o->ev_join[k];
      o->stream2[k] = nullptr;
      o->ev_join[k] = nullptr;
    }
    h->gexec = o->gexec;   // re-captured and updated in place at the first interval
    o->gexec = nullptr;
    h->graph_tile = -1;
    if (o->pinned_cap >= h->nrep) {
      h->hT = o->hT; h->hP = o->hP; h->havg = o->havg;
      h->pinned_cap = o->pinned_cap;
      o->hT = o->hP = o->havg = nullptr;
      o->pinned_cap = 0;
    }
    if (cudaSetDevice(device) != cudaSuccess || force_kernel_setup() != cudaSuccess) {
      set_error("cannot set up device");
      undo_carry(h, cy);
      return REMD_ERR_CUDA;
    }
  } else {
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        force_kernel_setup() != cudaSuccess) {
      set_error("cannot set up device/stream");
      delete h;
      return REMD_ERR_CUDA;
    }
    for (int k = 0; k < kMaxChains - 1; k++)
      if (cudaStreamCreateWithFlags(&h->stream2[k], cudaStreamNonBlocking) != cudaSuccess ||
          cudaEventCreateWithFlags(&h->ev_join[k], cudaEventDisableTiming) != cudaSuccess) {
        set_error("cannot create the interval graph's streams");
        undo_carry(h, cy);
        return REMD_ERR_CUDA;
      }
  }
  remd_status st = allocate(h);
  if (st != REMD_OK) { undo_carry(h, cy); return st; }
  // host SoA staging
  const int N = h->N;
  std::vector<double> r((size_t)N * 3), v((size_t)N * 3), q((size_t)N * 4), p((size_t)N * 4);
  for (int k = 0; k < h->nrep; k++) {
    if (cy && cy->from && cy->src_rep[k] >= 0) continue;   // copied on the device below
    const remd_replica_init& ri = reps[k];
    const RepConst& c = h->rc[k];
    for (int i = 0; i < c.nmol; i++) {
      const int g = c.mol_off + i;
      for (int x = 0; x < 3; x++) { r[(size_t)x * N + g] = ri.r[3 * i + x]; v[(size_t)x * N + g] = ri.v[3 * i + x]; }
      for (int x = 0; x < 4; x++) { q[(size_t)x * N + g] = ri.q[4 * i + x]; p[(size_t)x * N + g] = ri.p[4 * i + x]; }
    }
  }
  if ((st = upload_state(h, r, v, q, p, st0)) != REMD_OK) { undo_carry(h, cy); return st; }
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) { set_error("state upload failed"); undo_carry(h, cy); return REMD_ERR_CUDA; }
  if (!h->hT) {
    if (cudaMallocHost(&h->hT, h->nrep * 8) != cudaSuccess || cudaMallocHost(&h->hP, h->nrep * 8) != cudaSuccess ||
        cudaMallocHost(&h->havg, (size_t)h->nrep * kNumAvg * 8) != cudaSuccess) {
      set_error("pinned host allocation failed");
      undo_carry(h, cy);
      return REMD_ERR_OOM;
    }
    h->pinned_cap = h->nrep;
  }
  // device-side exchange bookkeeping: identity index, current conditions
  {
    std::vector<int> idx(h->nrep), grid(2 * nens), roff(nens), uoff(nens);
    for (int e = 0; e < nens; e++) {
      roff[e] = h->ens_rep_off[e];
      for (int k = 0; k < h->ens_nrep[e]; k++) idx[roff[e] + k] = k;
    }
    if (cudaMemcpy(h->d_index, idx.data(), idx.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(h->dT, h->curT.data(), h->nrep * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(h->dP, h->curP.data(), h->nrep * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(h->d_rep_off, roff.data(), roff.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
      set_error("upload of the condition arrays failed");
      undo_carry(h, cy);
      return REMD_ERR_CUDA;
    }
  }
  if (cy) st = carry_in(h, cy);
  else st = initial_force(h);
  if (st != REMD_OK) { undo_carry(h, cy); return st; }
  h->last_pairs = host_pairs(h);
  *out = h;
  return REMD_OK;
}

extern "C" {

remd_status remd_create(const remd_system_desc* systems, int nens, const int* reps_per_ens,
                        const remd_replica_init* reps, remd_precision prec, int device,
                        remd_handle* out) {
  return create_impl(systems, nens, reps_per_ens, reps, prec, device, nullptr, out);
}

remd_status remd_destroy(remd_handle h) {
  if (!h) return REMD_OK;
  if (h->gexec) cudaGraphExecDestroy(h->gexec);
  if (h->pool) free_pool(h);
  if (h->hT) cudaFreeHost(h->hT);
  if (h->hP) cudaFreeHost(h->hP);
  if (h->havg) cudaFreeHost(h->havg);
  for (auto& H : h->hist) {
    if (H.hist) cudaFree(H.hist);
    if (H.ave) cudaFree(H.ave);
    if (H.bounds) cudaFree(H.bounds);
  }
  if (h->d_hist) cudaFree(h->d_hist);
  if (h->d_hidx) cudaFree(h->d_hidx);
  if (h->ev_fork) cudaEventDestroy(h->ev_fork);
  for (int k = 0; k < kMaxChains - 1; k++) {
    if (h->ev_join[k]) cudaEventDestroy(h->ev_join[k]);
    if (h->stream2[k]) cudaStreamDestroy(h->stream2[k]);
  }
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return REMD_OK;
}

// Everything a re-layout must carry: the molecule and replica state, the
// conditions and index, and the device-exchange configuration.
struct SavedState {
  std::vector<double> r, v, q, p, dT, dP;
  std::vector<RepState> st;
  std::vector<int> idx, grid, uoff;
  std::vector<long long> step;
  std::vector<unsigned long long> seed;
};

static remd_status save_state(remd_engine_s* h, SavedState& sv) {
  const int N = h->N;
  sv.r.resize((size_t)N * 3); sv.v.resize((size_t)N * 3); sv.q.resize((size_t)N * 4); sv.p.resize((size_t)N * 4);
  sv.st.resize(h->nrep); sv.dT.resize(h->nrep); sv.dP.resize(h->nrep); sv.idx.resize(h->nrep);
  sv.grid.resize(2 * h->nens); sv.uoff.resize(h->nens); sv.step.resize(h->nens); sv.seed.resize(h->nens);
  CK(cudaStreamSynchronize(h->stream));
  CK(cudaMemcpy(sv.r.data(), h->d.r, sv.r.size() * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(sv.v.data(), h->d.v, sv.v.size() * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(sv.q.data(), h->d.q, sv.q.size() * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(sv.p.data(), h->d.p, sv.p.size() * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(sv.st.data(), h->X, sv.st.size() * sizeof(RepState), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(sv.dT.data(), h->dT, h->nrep * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(sv.dP.data(), h->dP, h->nrep * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(sv.idx.data(), h->d_index, h->nrep * 4, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(sv.grid.data(), h->d_grid, sv.grid.size() * 4, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(sv.uoff.data(), h->d_u_off, sv.uoff.size() * 4, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(sv.step.data(), h->d_step, sv.step.size() * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(sv.seed.data(), h->d_seed, sv.seed.size() * 8, cudaMemcpyDeviceToHost));
  return REMD_OK;
}

// Re-lay out the arrays for (tile, skin) and restore `sv`.  Forces are a pure
// function of the positions and every partial sum is per 32 molecules, so the
// trajectory that follows does not depend on the tile or the skin.
static remd_status relayout(remd_engine_s* h, int tile, double skin, const SavedState& sv) {
  h->tile = tile;
  h->skin = skin;
  for (auto& c : h->rc) {
    c.skin = skin;
    const double rl = c.rc + skin;
    const double cap = 0.1 * 4.0 / 3.0 * M_PI * rl * rl * rl;
    c.nbr_cap = std::max(1, std::min(c.nmol - 1, ((int)std::ceil(cap) + 7) / 8 * 8));
  }
  if (h->gexec) { cudaGraphExecDestroy(h->gexec); h->gexec = nullptr; }
  remd_status s = allocate(h);
  if (s != REMD_OK) return s;
  if ((s = upload_state(h, sv.r, sv.v, sv.q, sv.p, sv.st)) != REMD_OK) return s;
  CK(cudaStreamSynchronize(h->stream));
  std::vector<int> roff(h->nens);
  for (int e = 0; e < h->nens; e++) roff[e] = h->ens_rep_off[e];
  CK(cudaMemcpy(h->dT, sv.dT.data(), h->nrep * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->dP, sv.dP.data(), h->nrep * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->d_index, sv.idx.data(), h->nrep * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->d_rep_off, roff.data(), roff.size() * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->d_grid, sv.grid.data(), sv.grid.size() * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->d_u_off, sv.uoff.data(), sv.uoff.size() * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->d_step, sv.step.data(), sv.step.size() * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->d_seed, sv.seed.data(), sv.seed.size() * 8, cudaMemcpyHostToDevice));
  // forces are a pure function of positions: recompute, keep H0
  launch_pack(h->d, h->prec, h->tile, h->stream);
  launch_force(h->d, h->X, h->X, h->prec, true, h->tile, h->stream);
  CK(cudaGetLastError());
  return sync_and_check(h);
}

remd_status remd_set_tuning(remd_handle h, int tile, double skin) {
  if (!h || tile < 32 || tile > max_force_tile(h->prec) || tile % 32 || !(skin > 0.0)) {
    set_error("remd_set_tuning: tile must be a multiple of 32 in 32..64 (FP32) or 32..128 (FP64), skin > 0");
    return REMD_ERR_INVALID;
  }
  if (tile == h->tile && skin == h->skin) return REMD_OK;
  SavedState sv;
  remd_status s = save_state(h, sv);
  if (s != REMD_OK) return s;
  return relayout(h, tile, skin, sv);
}

remd_status remd_autotune(remd_handle h, int nsteps, int* tile_out, double* skin_out, double* ms_out) {
  if (!h || nsteps < 1) return REMD_ERR_INVALID;
  SavedState sv;
  remd_status s = save_state(h, sv);
  if (s != REMD_OK) return s;
  const long long steps0 = h->steps_done;   // the trials' steps are undone with the state
  static const int tiles[] = {32, 64, 96, 128};
  static const double skins[] = {0.2, 0.4, 0.6, 0.8, 1.0, 1.4};
  int best_tile = h->tile;
  double best_skin = h->skin, best_ms = 1e300;
  for (int t : tiles)
    for (double k : skins) {
      if (t > max_force_tile(h->prec)) continue;
      if ((s = relayout(h, t, k, sv)) != REMD_OK) return s;
      double ms[2];
      if ((s = remd_profile_steps(h, nsteps, ms)) != REMD_OK) return s;
      const double step_ms = ms[0] + ms[1];
      if (step_ms < best_ms) { best_ms = step_ms; best_tile = t; best_skin = k; }
    }
  if ((s = relayout(h, best_tile, best_skin, sv)) != REMD_OK) return s;
  h->steps_done = steps0;
  if (tile_out) *tile_out = best_tile;
  if (skin_out) *skin_out = best_skin;
  if (ms_out) *ms_out = best_ms;
  return REMD_OK;
}

remd_status remd_execute_steps_async(remd_handle h, const double* T, const double* P) {
  if (!h) { set_error("null handle"); return REMD_ERR_INVALID; }
  if (T && P) {
    for (int k = 0; k < h->nrep; k++) {
      if (!(T[k] > 0.0)) { set_error("temperatures must be > 0"); return REMD_ERR_INVALID; }
      h->hT[k] = T[k];
      h->hP[k] = P[k];
    }
    CK(cudaMemcpyAsync(h->dT, h->hT, h->nrep * 8, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->dP, h->hP, h->nrep * 8, cudaMemcpyHostToDevice, h->stream));
  }
  if (!h->gexec || h->graph_tile != h->tile || h->graph_exchange != h->exch_enabled ||
      h->graph_hist != h->hist_on) {
    const auto g0 = std::chrono::steady_clock::now();
    remd_status s = build_graph(h);
    h->last_graph_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - g0).count();
    if (s != REMD_OK) return s;
  } else {
    h->last_graph_ms = 0.0;
  }
  CK(cudaGraphLaunch(h->gexec, h->stream));
  h->steps_done += h->interval;
  return REMD_OK;
}

remd_status remd_synchronize(remd_handle h) {
  if (!h) return REMD_ERR_INVALID;
  return sync_and_check(h);
}

remd_status remd_execute_steps(remd_handle h, const double* T, const double* P) {
  if (!h || !T || !P) { set_error("remd_execute_steps: null argument"); return REMD_ERR_INVALID; }
  remd_status s = remd_execute_steps_async(h, T, P);
  if (s != REMD_OK) return s;
  CK(cudaMemcpyAsync(h->havg, h->d.avg, (size_t)h->nrep * kNumAvg * 8, cudaMemcpyDeviceToHost, h->stream));
  s = sync_and_check(h);
  for (int k = 0; k < h->nrep; k++) { h->curT[k] = T[k]; h->curP[k] = P[k]; }
  return s;
}

remd_status remd_execute_steps_device(remd_handle h) {
  remd_status s = remd_execute_steps_async(h, nullptr, nullptr);
  if (s != REMD_OK) return s;
  CK(cudaMemcpyAsync(h->havg, h->d.avg, (size_t)h->nrep * kNumAvg * 8, cudaMemcpyDeviceToHost, h->stream));
  return sync_and_check(h);
}

remd_status remd_execute_nsteps(remd_handle h, int nsteps) {
  if (!h || nsteps < 1) { set_error("remd_execute_nsteps: nsteps must be >= 1"); return REMD_ERR_INVALID; }
  launch_replica_start(h->d, h->X, h->stream);
  for (int s = 0; s < nsteps; s++) {
    launch_step_integrate(h, s);
    launch_force(h->d, h->Y, h->X, h->prec, false, h->tile, h->stream);
  }
  launch_replica_end(h->d, h->X, h->stream);
  CK(cudaGetLastError());
  h->steps_done += nsteps;
  return sync_and_check(h);
}

remd_status remd_rescale_velocities(remd_handle h) {
  if (!h) return REMD_ERR_INVALID;
  launch_replica_rescale(h->d, h->X, false, h->stream);
  CK(cudaGetLastError());
  return sync_and_check(h);
}

remd_status remd_get_averages(remd_handle h, int rep, double* out) {
  if (!h || !out || rep < 0 || rep >= h->nrep) { set_error("remd_get_averages: bad argument"); return REMD_ERR_INVALID; }
  CK(cudaStreamSynchronize(h->stream));
  CK(cudaMemcpy(out, h->d.avg + (size_t)rep * kNumAvg, kNumAvg * 8, cudaMemcpyDeviceToHost));
  return REMD_OK;
}

remd_status remd_get_all_averages(remd_handle h, double* out) {
  if (!h || !out) { set_error("remd_get_all_averages: bad argument"); return REMD_ERR_INVALID; }
  CK(cudaStreamSynchronize(h->stream));
  CK(cudaMemcpy(out, h->d.avg, (size_t)h->nrep * kNumAvg * 8, cudaMemcpyDeviceToHost));
  return REMD_OK;
}

remd_status remd_get_state(remd_handle h, int rep, remd_state_view* o) {
  if (!h || !o || rep < 0 || rep >= h->nrep) { set_error("remd_get_state: bad argument"); return REMD_ERR_INVALID; }
  CK(cudaStreamSynchronize(h->stream));
  const RepConst& c = h->rc[rep];
  const int n = c.nmol, N = h->N;
  std::vector<double> tmp((size_t)n);
  auto pull = [&](const double* src, int ncomp, double* dst) -> remd_status {
    if (!dst) return REMD_OK;
    for (int x = 0; x < ncomp; x++) {
      CK(cudaMemcpy(tmp.data(), src + (size_t)x * N + c.mol_off, n * 8, cudaMemcpyDeviceToHost));
      for (int i = 0; i < n; i++) dst[(size_t)ncomp * i + x] = tmp[i];
    }
    return REMD_OK;
  };
  remd_status s;
  if ((s = pull(h->d.r, 3, o->r)) != REMD_OK) return s;
  if ((s = pull(h->d.v, 3, o->v)) != REMD_OK) return s;
  if ((s = pull(h->d.q, 4, o->q)) != REMD_OK) return s;
  if ((s = pull(h->d.p, 4, o->p)) != REMD_OK) return s;
  if ((s = pull(h->d.f, 3, o->f)) != REMD_OK) return s;
  if ((s = pull(h->d.n, 4, o->n)) != REMD_OK) return s;
  RepState st;
  CK(cudaMemcpy(&st, h->X + rep, sizeof(st), cudaMemcpyDeviceToHost));
  o->s = st.s; o->Ps = st.Ps; o->Q = c.Q; o->W = c.W;
  for (int x = 0; x < 3; x++) { o->Pv[x] = st.Pv[x]; o->L[x] = st.L[x]; }
  o->T = st.T; o->P = st.P; o->H0 = st.H0;
  std::vector<Part2> p2(c.nwarp);
  CK(cudaMemcpy(p2.data(), h->d.part2 + c.warp_off, c.nwarp * sizeof(Part2), cudaMemcpyDeviceToHost));
  double lj = 0, cl = 0, w = 0, v[3] = {0, 0, 0};
  for (auto& p : p2) { lj += p.lj; cl += p.clmb; w += p.wall; for (int x = 0; x < 3; x++) v[x] += p.vir[x]; }
  o->lj = lj * 0.5; o->clmb = cl * 0.5; o->wall = w;
  for (int x = 0; x < 3; x++) o->vir[x] = v[x] * 0.5;
  o->pot = o->lj + o->clmb + o->wall;
  return REMD_OK;
}

remd_status remd_compute_forces(remd_handle h) {
  if (!h) return REMD_ERR_INVALID;
  launch_pack(h->d, h->prec, h->tile, h->stream);
  launch_force(h->d, h->X, h->X, h->prec, true, h->tile, h->stream);
  CK(cudaGetLastError());
  remd_status s = sync_and_check(h);
  h->last_pairs = host_pairs(h);
  return s;
}

int remd_num_replicas(remd_handle h) { return h ? h->nrep : 0; }
int remd_replica_nmol(remd_handle h, int rep) { return (h && rep >= 0 && rep < h->nrep) ? h->rc[rep].nmol : 0; }
long long remd_last_pair_count(remd_handle h) {
  if (!h) return -1;
  cudaStreamSynchronize(h->stream);
  h->last_pairs = host_pairs(h);
  return h->last_pairs;
}
int remd_launches_per_interval(remd_handle h) {
  // replica_start + per MD step (integrate, replica head, force: lists + pairs in FP32, one launch in FP64;
  // with velocity scaling also the rescale and, after the first step, the closing kick)
  // + replica_end + the device exchange when enabled (and the histogram before it)
  if (!h) return 0;
  // (the multi-chain graph, without velocity scaling, launches each step kernel once per chain)
  const int chains = h->vscale ? 1 : h->nchain;
  const int per_step = ((h->prec == kF32 ? 4 : 3) + (h->vscale ? 1 : 0)) * chains;
  return per_step * h->interval + (h->vscale ? h->interval - 1 : 0) + 2 + (h->exch_enabled ? 1 : 0) +
         (h->exch_enabled && h->hist_on ? 1 : 0);
}

long long remd_replica_pair_count(remd_handle h, int rep) {
  if (!h || rep < 0 || rep >= h->nrep) return -1;
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return -1;
  const RepConst& c = h->rc[rep];
  std::vector<Part2> p2(c.nwarp);
  if (cudaMemcpy(p2.data(), h->d.part2 + c.warp_off, c.nwarp * sizeof(Part2), cudaMemcpyDeviceToHost) != cudaSuccess)
    return -1;
  long long s = 0;
  for (auto& p : p2) s += p.npairs;
  return s / 2;
}

void* remd_stream(remd_handle h) { return h ? (void*)h->stream : nullptr; }

remd_status remd_profile_steps(remd_handle h, int nsteps, double* ms_out) {
  if (!h || nsteps < 1 || !ms_out) return REMD_ERR_INVALID;
  cudaEvent_t ev[3];
  for (auto& e : ev) CK(cudaEventCreate(&e));
  double ti = 0.0, tf = 0.0;
  for (int s = 0; s < nsteps; s++) {
    CK(cudaEventRecord(ev[0], h->stream));
    launch_step_integrate(h, s);
    CK(cudaEventRecord(ev[1], h->stream));
    launch_force(h->d, h->Y, h->X, h->prec, false, h->tile, h->stream);
    CK(cudaEventRecord(ev[2], h->stream));
    CK(cudaEventSynchronize(ev[2]));
    float a = 0.f, b = 0.f;
    CK(cudaEventElapsedTime(&a, ev[0], ev[1]));
    CK(cudaEventElapsedTime(&b, ev[1], ev[2]));
    ti += a;
    tf += b;
  }
  launch_replica_end(h->d, h->X, h->stream);
  for (auto& e : ev) cudaEventDestroy(e);
  h->steps_done += nsteps;
  ms_out[0] = ti / nsteps;
  ms_out[1] = tf / nsteps;
  return sync_and_check(h);
}

remd_status remd_profile_split(remd_handle h, int nsteps, double* ms_out) {
  if (!h || nsteps < 1 || !ms_out) return REMD_ERR_INVALID;
  cudaEvent_t ev[5];
  for (auto& e : ev) CK(cudaEventCreate(&e));
  double t[4] = {0, 0, 0, 0}, rebuilt = 0.0;
  std::vector<CellGrid> g(h->nrep);
  for (int s = 0; s < nsteps; s++) {
    CK(cudaEventRecord(ev[0], h->stream));
    launch_step_integrate(h, s);
    CK(cudaEventRecord(ev[1], h->stream));
    launch_force_timed(h->d, h->Y, h->X, h->prec, h->tile, h->stream, ev[2], ev[3]);
    CK(cudaEventRecord(ev[4], h->stream));
    CK(cudaEventSynchronize(ev[4]));
    for (int k = 0; k < 4; k++) {
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
      t[k] += ms;
    }
    CK(cudaMemcpy(g.data(), h->d.cgrid, h->nrep * sizeof(CellGrid), cudaMemcpyDeviceToHost));
    for (const CellGrid& x : g) rebuilt += x.rebuild ? 1.0 : 0.0;
  }
  launch_replica_end(h->d, h->X, h->stream);
  for (auto& e : ev) cudaEventDestroy(e);
  h->steps_done += nsteps;
  for (int k = 0; k < 4; k++) ms_out[k] = t[k] / nsteps;
  ms_out[4] = rebuilt / nsteps;
  return sync_and_check(h);
}

remd_status remd_measure_fp32_peak(int device, double* tflops) {
  if (!tflops) return REMD_ERR_INVALID;
  CK(cudaSetDevice(device));
  double ms = 0.0;
  long long flops = 0;
  remd_status s = (remd_status)measure_fp32_fma(device, &ms, &flops);
  if (s != REMD_OK) return s;
  *tflops = (double)flops / (ms * 1e-3) / 1e12;
  return REMD_OK;
}

remd_status remd_measure_atomics(int device, double* rates) {
  if (!rates) return REMD_ERR_INVALID;
  CK(cudaSetDevice(device));
  const int s = measure_atomics(device, rates);
  if (s != 0) { set_error("atomic throughput probe failed"); return (remd_status)s; }
  return REMD_OK;
}

remd_status remd_replica_status(remd_handle h, int rep, int* status) {
  if (!h || !status || rep < 0 || rep >= h->nrep) return REMD_ERR_INVALID;
  CK(cudaMemcpy(status, h->d.status + rep, 4, cudaMemcpyDeviceToHost));
  return REMD_OK;
}

remd_status remd_exchange_device(remd_handle h, const int* grids, long step, const double* u,
                                 unsigned long long seed) {
  if (!h || !grids) { set_error("remd_exchange_device: null argument"); return REMD_ERR_INVALID; }
  std::vector<int> uoff(h->nens);
  int tot = 0;
  for (int e = 0; e < h->nens; e++) {
    if (grids[2 * e] * grids[2 * e + 1] != h->ens_nrep[e]) {
      set_error("exchange grid does not match the replica count of ensemble " + std::to_string(e));
      return REMD_ERR_INVALID;
    }
    uoff[e] = tot;
    tot += exchange_pair_count(grids[2 * e], grids[2 * e + 1], step);
  }
  CK(cudaMemcpyAsync(h->d_grid, grids, 2 * h->nens * 4, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_u_off, uoff.data(), h->nens * 4, cudaMemcpyHostToDevice, h->stream));
  const double* du = nullptr;
  if (u) {
    if (tot > h->u_cap) { set_error("too many uniforms"); return REMD_ERR_INVALID; }
    if (tot > 0) CK(cudaMemcpyAsync(h->d_u, u, tot * 8, cudaMemcpyHostToDevice, h->stream));
    du = h->d_u;
  }
  {
    std::vector<unsigned long long> sd(h->nens, seed);
    CK(cudaMemcpyAsync(h->d_seed, sd.data(), h->nens * 8, cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
  }
  launch_exchange_k(h->d, h->d_grid, h->d_rep_off, h->d_u_off, h->nens, step, du, h->d_seed, h->d_index,
                    h->dT, h->dP, h->d_step, h->stream);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(h->stream));   // host arrays (uoff) go out of scope
  return REMD_OK;
}

remd_status remd_enable_device_exchange(remd_handle h, const int* grids, unsigned long long seed,
                                        long long first_step) {
  if (!h) return REMD_ERR_INVALID;
  if (!grids) {
    h->exch_enabled = false;
    return REMD_OK;
  }
  for (int e = 0; e < h->nens; e++)
    if (grids[2 * e] < 1 || grids[2 * e + 1] < 1 || grids[2 * e] * grids[2 * e + 1] != h->ens_nrep[e]) {
      set_error("exchange grid does not match the replica count of ensemble " + std::to_string(e));
      return REMD_ERR_INVALID;
    }
  std::vector<long long> st(h->nens, first_step);
  std::vector<unsigned long long> sd(h->nens, seed);
  CK(cudaMemcpyAsync(h->d_grid, grids, 2 * h->nens * 4, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_step, st.data(), h->nens * 8, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_seed, sd.data(), h->nens * 8, cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  h->exch_enabled = true;
  h->exch_seed = seed;
  return REMD_OK;
}

remd_status remd_get_conditions(remd_handle h, int* index, double* T, double* P) {
  if (!h) return REMD_ERR_INVALID;
  CK(cudaStreamSynchronize(h->stream));
  if (index) CK(cudaMemcpy(index, h->d_index, h->nrep * 4, cudaMemcpyDeviceToHost));
  if (T) CK(cudaMemcpy(T, h->dT, h->nrep * 8, cudaMemcpyDeviceToHost));
  if (P) CK(cudaMemcpy(P, h->dP, h->nrep * 8, cudaMemcpyDeviceToHost));
  return REMD_OK;
}

remd_status remd_write_chk(remd_handle h, int rep, const char* path) {
  if (!h || !path || rep < 0 || rep >= h->nrep) return REMD_ERR_INVALID;
  const RepConst& c = h->rc[rep];
  const int n = c.nmol;
  std::vector<double> r(3 * n), v(3 * n), q(4 * n), p(4 * n);
  remd_state_view o;
  std::memset(&o, 0, sizeof(o));
  o.r = r.data(); o.v = v.data(); o.q = q.data(); o.p = p.data();
  remd_status s = remd_get_state(h, rep, &o);
  if (s != REMD_OK) return s;
  double a[kNumAvg];
  if ((s = remd_get_averages(h, rep, a)) != REMD_OK) return s;
  // the Property line (Molecules::CalcProperties, src/molecules.cxx:702-734)
  double prop[kChkPropCount];
  double t = 0.0;   // prop.time += unit_time * dt once per MD step (src/integrator.cxx:795)
  for (long long k = 0; k < h->steps_done; k++) t += unit_time() * c.dt;
  const double gkT = 6.0 * (double)n * o.T;
  const double tsm = 0.5 * o.Ps * o.Ps / o.Q, tsp = gkT * std::log(o.s);
  double bst = 0.0;   // Molecules::BarostatEnergy (src/molecules.cxx:663-678); slit: GPU form
  if (c.pconstant > 0) {
    if (c.confined == 0)
      bst = 0.5 * (o.Pv[0] * o.Pv[0] + o.Pv[1] * o.Pv[1] + o.Pv[2] * o.Pv[2]) / c.W + o.P * o.L[0] * o.L[1] * o.L[2];
    else if (c.confined == 1)
      bst = 0.5 * o.Pv[2] * o.Pv[2] / c.W + o.P * (c.bottom_area * o.L[2]);
    else
      bst = (o.Pv[0] * o.Pv[0] + o.Pv[1] * o.Pv[1]) * (0.5 / c.W) + o.P * (o.L[0] * o.L[1] * c.slit_width);
  }
  double tmo[3] = {0.0, 0.0, 0.0};   // Molecules::Momentum (src/molecules.cxx:679-686)
  for (int x = 0; x < 3; x++) {
    const double cf = 1.0 / (o.L[x] * o.s);
    for (int i = 0; i < n; i++) tmo[x] += v[3 * i + x] * c.mass * cf;
  }
  const double up = unit_press();
  const double prs[4] = {a[REMD_AVG_PX] * up, a[REMD_AVG_PY] * up, a[REMD_AVG_PZ] * up, a[REMD_AVG_P] * up};
  const double vals[kChkPropCount] = {
      t, a[0] + a[1] + a[2], a[REMD_AVG_TRA], a[REMD_AVG_ROT], a[REMD_AVG_TRA] + a[REMD_AVG_ROT], tsm, tsp,
      tsm + tsp, bst, a[REMD_AVG_TOT], a[REMD_AVG_DRF], tmo[0], tmo[1], tmo[2], a[REMD_AVG_T] * unit_temp(),
      prs[0], prs[1], prs[2], prs[3], o.vir[0], o.vir[1], o.vir[2], prs[0], prs[1], prs[2], prs[3]};
  std::memcpy(prop, vals, sizeof(prop));
  return (remd_status)write_chk(path, n, c.nsite, r.data(), v.data(), q.data(), p.data(), c.mass, c.I,
                                o.s, o.Ps, o.Q, o.Pv, o.W, o.L, prop);
}

remd_status remd_write_gro(remd_handle h, int rep, const char* path, const char* mol_name,
                           const char* const* atom_names) {
  if (!h || !path || !mol_name || !atom_names || rep < 0 || rep >= h->nrep) return REMD_ERR_INVALID;
  const RepConst& c = h->rc[rep];
  const int n = c.nmol, ns = c.nsite;
  for (int k = 0; k < ns; k++)
    if (!atom_names[k]) return REMD_ERR_INVALID;
  std::vector<double> r(3 * n), q(4 * n);
  remd_state_view o;
  std::memset(&o, 0, sizeof(o));
  o.r = r.data(); o.q = q.data();
  remd_status s = remd_get_state(h, rep, &o);
  if (s != REMD_OK) return s;
  // names as MakeMolTypeList pads them (src/molecules.cxx:86, 95): the molecule
  // name left-justified, the atom names right-justified, to 5 characters
  std::string mname(mol_name);
  while (mname.size() < 5) mname += " ";
  std::vector<std::string> anames(ns);
  for (int k = 0; k < ns; k++) {
    anames[k] = atom_names[k];
    while (anames[k].size() < 5) anames[k] = " " + anames[k];
  }
  FILE* fp = std::fopen(path, "w");
  if (!fp) {
    set_error(std::string("remd_write_gro: cannot open ") + path);
    return REMD_ERR_IO;
  }
  // IOManager::ConvertMoleculesToAtoms (src/io_manager.cxx:797-814): site = r L + R(q) b,
  // angstrom -> nm, velocities written as zero; write_gro_file (src/gro.cxx:118-135)
  // with the comment and the box in nm of IOManager::UpdateOutputs (src/io_manager.cxx:636-651)
  const double A_to_nm = 0.1;
  std::fprintf(fp, "%s\n", "test");
  std::fprintf(fp, "%5d\n", n * ns);
  int count = 0;
  for (int i = 0; i < n; i++) {
    const double qi[4] = {q[4 * i], q[4 * i + 1], q[4 * i + 2], q[4 * i + 3]};
    for (int k = 0; k < ns; k++) {
      double sk[3];
      body_to_space(qi, c.body[k], sk);
      double x[3];
      for (int d = 0; d < 3; d++) x[d] = (r[3 * i + d] * o.L[d] + sk[d]) * A_to_nm;
      count++;
      std::fprintf(fp, "%5d%s%s%5d%8.3lf%8.3lf%8.3lf%8.4lf%8.4lf%8.4lf\n", i + 1, mname.c_str(),
                   anames[k].c_str(), count, x[0], x[1], x[2], 0.0, 0.0, 0.0);
    }
  }
  std::fprintf(fp, "%10.5lf%10.5lf%10.5lf\n", o.L[0] * A_to_nm, o.L[1] * A_to_nm, o.L[2] * A_to_nm);
  const bool ok = std::fclose(fp) == 0;
  if (!ok) {
    set_error(std::string("remd_write_gro: write failed: ") + path);
    return REMD_ERR_IO;
  }
  return REMD_OK;
}

// REMDGPU::OutputCDV (src/remdgpu.cu:700-804): one CDView snapshot per replica,
// <prefix>R<rep, 4 digits>s<step, 7 digits>.cdv.  The numbers are the ones that
// the reference's GPU state holds and prints: the centre of mass as a 32-bit
// fixed-point box fraction (int)(2^32 (r - 1/2)), the box and the wall length
// in single precision, the site offsets R(q) b rounded to float, each site
// printed as float(centre * (L 2^-32)) + offset; the condition as the float it
// keeps (cond0), in K and MPa.  Text formatting is the C++ stream default
// (6 significant digits), as in the reference.
remd_status remd_output_cdv(remd_handle h, const char* prefix, unsigned int step) {
  if (!h || !prefix) return REMD_ERR_INVALID;
  const float to_frac = (float)kFixInv;   // 2^-32, exact in float
  for (int rep = 0; rep < h->nrep; rep++) {
    const RepConst& c = h->rc[rep];
    const int n = c.nmol, ns = c.nsite;
    std::vector<double> r(3 * n), q(4 * n);
    remd_state_view o;
    std::memset(&o, 0, sizeof(o));
    o.r = r.data(); o.q = q.data();
    remd_status st = remd_get_state(h, rep, &o);
    if (st != REMD_OK) return st;
    std::ostringstream name;
    name << prefix << "R" << std::setw(4) << std::setfill('0') << rep << "s" << std::setw(7)
         << std::setfill('0') << step << ".cdv";
    std::ofstream os(name.str());
    if (!os) {
      set_error("remd_output_cdv: cannot open " + name.str());
      return REMD_ERR_IO;
    }
    const float L[3] = {(float)o.L[0], (float)o.L[1], (float)o.L[2]};
    const float wl = (float)c.wall_length_param;
    const float ItoF[3] = {L[0] * to_frac, L[1] * to_frac, L[2] * to_frac};
    os << "'";
    double lo[3], hi[3];
    for (int d = 0; d < 3; d++) { lo[d] = -0.5 * L[d]; hi[d] = 0.5 * L[d]; }
    if (c.confined == 1) { lo[0] = lo[1] = -wl; hi[0] = hi[1] = wl; }
    if (c.confined == 2) { lo[2] = -0.5 * wl; hi[2] = 0.5 * wl; }
    os << " box_sx=" << lo[0] << " box_sy=" << lo[1] << " box_sz=" << lo[2];
    os << " box_ex=" << hi[0] << " box_ey=" << hi[1] << " box_ez=" << hi[2];
    // site radii and colours (oxygen red, the rest white) and the condition label
    os << " r0=1.0 r1=0.8 r2=0.8 c0=(1.0,0.0,0.0) c1=(1.0,1.0,1.0) c2=(1.0,1.0,1.0)"
          " bond0_c=(1.0,1.0,1.0)";
    const double T = (double)(float)o.T * unit_temp(), P = (double)(float)o.P * unit_press();
    os << " st0=\"T=" << T << " K, P=" << P / 1e6 << " MPa\" st0_pos=(-2.0,-2.0)\n";
    for (int i = 0; i < n; i++) {
      int g[3];
      for (int d = 0; d < 3; d++) g[d] = (int)(kFix * (r[3 * i + d] - 0.5));
      const double qi[4] = {q[4 * i], q[4 * i + 1], q[4 * i + 2], q[4 * i + 3]};
      for (int k = 0; k < ns; k++) {
        const double b[3] = {(double)(float)c.body[k][0], (double)(float)c.body[k][1],
                             (double)(float)c.body[k][2]};
        double sk[3];
        body_to_space(qi, b, sk);
        os << i << " " << k;
        for (int d = 0; d < 3; d++) {
          const float a = (float)g[d] * ItoF[d] + (float)sk[d];
          os << " " << a;
        }
        os << "\n";
      }
    }
    os.close();
    if (!os) {
      set_error("remd_output_cdv: write failed: " + name.str());
      return REMD_ERR_IO;
    }
  }
  return REMD_OK;
}

// ---- histograms (REMDInfo's Histogram, src/remdinfo.h:93-139, 299-331) ----

remd_status remd_histogram_enable(remd_handle h, int ens, double energy_min, double energy_max,
                                  double volume_min, double volume_max) {
  if (!h || ens < 0 || ens >= h->nens || !(energy_max > energy_min) || !(volume_max > volume_min)) {
    set_error("remd_histogram_enable: need a valid ensemble and max > min");
    return REMD_ERR_INVALID;
  }
  CK(cudaSetDevice(h->device));
  CK(cudaStreamSynchronize(h->stream));
  if (!h->d_hist) {
    CK(cudaMalloc(&h->d_hist, sizeof(HistEns) * h->nens));
    CK(cudaMalloc(&h->d_hidx, sizeof(int) * h->nrep));
    h->hist.assign(h->nens, HistEns{});
    h->h_hidx.resize(h->nrep);
    for (int e = 0; e < h->nens; e++)
      for (int c = 0; c < h->ens_nrep[e]; c++) h->h_hidx[h->ens_rep_off[e] + c] = c;
  }
  HistEns& H = h->hist[ens];
  if (H.hist) { cudaFree(H.hist); cudaFree(H.ave); cudaFree(H.bounds); H = HistEns{}; }
  const size_t nc = (size_t)h->ens_nrep[ens];
  const size_t bins = nc * kHistBins * kHistBins;
  if (cudaMalloc(&H.hist, bins * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&H.ave, bins * kNumAvg * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&H.bounds, nc * 5 * sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    if (H.hist) cudaFree(H.hist);
    if (H.ave) cudaFree(H.ave);
    if (H.bounds) cudaFree(H.bounds);
    H = HistEns{};
    set_error("remd_histogram_enable: device allocation failed");
    return REMD_ERR_OOM;
  }
  CK(cudaMemset(H.hist, 0, bins * sizeof(int)));
  CK(cudaMemset(H.ave, 0, bins * kNumAvg * sizeof(double)));
  CK(cudaMemset(H.bounds, 0, nc * 5 * sizeof(int)));
  // REMDInfo::REMDInfo, linear sampling (src/remdinfo.cxx:180-186)
  H.emin = energy_min; H.emax = energy_max; H.de = (energy_max - energy_min) / (double)kHistBins;
  H.vmin = volume_min; H.vmax = volume_max; H.dv = (volume_max - volume_min) / (double)kHistBins;
  CK(cudaMemcpy(h->d_hist, h->hist.data(), sizeof(HistEns) * h->nens, cudaMemcpyHostToDevice));
  h->hist_on = true;
  return REMD_OK;
}

remd_status remd_histogram_increment(remd_handle h, const int* index) {
  if (!h || !h->hist_on) { set_error("remd_histogram_increment: no histogram enabled"); return REMD_ERR_INVALID; }
  const int* d_idx = h->d_index;
  if (index) {
    for (int e = 0; e < h->nens; e++)
      for (int c = 0; c < h->ens_nrep[e]; c++) {
        const int k = index[h->ens_rep_off[e] + c];
        if (k < 0 || k >= h->ens_nrep[e]) { set_error("remd_histogram_increment: index out of range"); return REMD_ERR_INVALID; }
      }
    std::copy(index, index + h->nrep, h->h_hidx.begin());
    CK(cudaMemcpyAsync(h->d_hidx, h->h_hidx.data(), h->nrep * 4, cudaMemcpyHostToDevice, h->stream));
    d_idx = h->d_hidx;
  }
  launch_histogram(h->d, h->d_hist, h->d_rep_off, d_idx, h->stream);
  CK(cudaGetLastError());
  return sync_and_check(h);
}

remd_status remd_histogram_get(remd_handle h, int ens, int slot, int* bounds, int* hist, double* ave) {
  if (!h || ens < 0 || ens >= h->nens || !h->hist_on || !h->hist[ens].hist || slot < 0 ||
      slot >= h->ens_nrep[ens]) {
    set_error("remd_histogram_get: no such histogram");
    return REMD_ERR_INVALID;
  }
  CK(cudaStreamSynchronize(h->stream));
  const HistEns& H = h->hist[ens];
  const size_t nb = (size_t)kHistBins * kHistBins;
  if (bounds) CK(cudaMemcpy(bounds, H.bounds + 5 * slot, 5 * sizeof(int), cudaMemcpyDeviceToHost));
  if (hist) CK(cudaMemcpy(hist, H.hist + nb * slot, nb * sizeof(int), cudaMemcpyDeviceToHost));
  if (ave) CK(cudaMemcpy(ave, H.ave + nb * kNumAvg * slot, nb * kNumAvg * sizeof(double), cudaMemcpyDeviceToHost));
  return REMD_OK;
}

// The condition of each slot of ensemble e as REMDInfo holds it
// (temperature[index[slot]], pressure[index[slot]]).
static remd_status slot_conditions(remd_engine_s* h, int e, std::vector<double>& Tc, std::vector<double>& Pc) {
  std::vector<int> idx(h->nrep);
  std::vector<double> T(h->nrep), P(h->nrep);
  CK(cudaStreamSynchronize(h->stream));
  // the conditions of the last interval (the device exchange updates them in place)
  CK(cudaMemcpy(T.data(), h->dT, h->nrep * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(P.data(), h->dP, h->nrep * 8, cudaMemcpyDeviceToHost));
  if (h->exch_enabled) CK(cudaMemcpy(idx.data(), h->d_index, h->nrep * 4, cudaMemcpyDeviceToHost));
  else idx = h->h_hidx;
  const int off = h->ens_rep_off[e], n = h->ens_nrep[e];
  Tc.resize(n);
  Pc.resize(n);
  for (int c = 0; c < n; c++) {
    Tc[c] = T[off + idx[off + c]];
    Pc[c] = P[off + idx[off + c]];
  }
  return REMD_OK;
}

static std::string histo_name(const char* dir, double P, double T) {
  char buf[1024];
  std::snprintf(buf, sizeof(buf), "%s/histo_P%lf_T%lf.dat", dir, P, T);
  return buf;
}

// REMDInfo::OutputHistogram (src/remdinfo.cxx:723-758), linear sampling.
remd_status remd_histogram_write(remd_handle h, int ens, const char* dir) {
  if (!h || !dir || ens < 0 || ens >= h->nens || !h->hist_on || !h->hist[ens].hist) {
    set_error("remd_histogram_write: no such histogram");
    return REMD_ERR_INVALID;
  }
  std::vector<double> Tc, Pc;
  remd_status st = slot_conditions(h, ens, Tc, Pc);
  if (st != REMD_OK) return st;
  const HistEns& H = h->hist[ens];
  const size_t nb = (size_t)kHistBins * kHistBins;
  std::vector<int> hist(nb);
  std::vector<double> ave(nb * kNumAvg);
  for (int c = 0; c < h->ens_nrep[ens]; c++) {
    int b[5];
    st = remd_histogram_get(h, ens, c, b, hist.data(), ave.data());
    if (st != REMD_OK) return st;
    const std::string path = histo_name(dir, Pc[c], Tc[c]);
    FILE* fp = std::fopen(path.c_str(), "w");
    if (!fp) { set_error("remd_histogram_write: cannot open " + path); return REMD_ERR_IO; }
    std::fprintf(fp, "#vmax vmin pmax pmin\n");
    std::fprintf(fp, "# %d %d %d %d\n", b[1], b[0], b[3], b[2]);
    for (int v = b[0]; v <= b[1]; v++) {
      const double vol = H.vmin + v * H.dv;
      for (int p = b[2]; p <= b[3]; p++) {
        const double pot = H.emin + p * H.de;
        const size_t bin = (size_t)v * kHistBins + p;
        const int n = hist[bin];
        std::fprintf(fp, " %10.6e %10.6e %10d", vol, pot, n);
        for (int x = 0; x < kNumAvg; x++)   // Histogram::GetAverages: sum / count, 0 if empty
          std::fprintf(fp, " %10.6e", n > 0 ? ave[bin * kNumAvg + x] / (double)n : 0.0);
        std::fprintf(fp, "\n");
      }
      std::fprintf(fp, "\n");
    }
    if (std::fclose(fp) != 0) { set_error("remd_histogram_write: write failed: " + path); return REMD_ERR_IO; }
  }
  return REMD_OK;
}

// REMDInfo::ReadHistogramFromBackUp (src/remdinfo.cxx:681-721): counts and the
// per-bin averages (times the count) of every slot, from the files
// remd_histogram_write (OutputHistogram) made.
remd_status remd_histogram_read(remd_handle h, int ens, const char* dir) {
  if (!h || !dir || ens < 0 || ens >= h->nens || !h->hist_on || !h->hist[ens].hist) {
    set_error("remd_histogram_read: no such histogram");
    return REMD_ERR_INVALID;
  }
  std::vector<double> Tc, Pc;
  remd_status st = slot_conditions(h, ens, Tc, Pc);
  if (st != REMD_OK) return st;
  const HistEns& H = h->hist[ens];
  const size_t nb = (size_t)kHistBins * kHistBins;
  std::vector<int> hist(nb);
  std::vector<double> ave(nb * kNumAvg);
  for (int c = 0; c < h->ens_nrep[ens]; c++) {
    const std::string path = histo_name(dir, Pc[c], Tc[c]);
    std::ifstream is(path);
    if (!is) { set_error("remd_histogram_read: input histogram file " + path + " is not found"); return REMD_ERR_IO; }
    std::string dummy;
    int b[5] = {0, 0, 0, 0, 0};
    is >> dummy >> dummy >> dummy >> dummy;
    is >> dummy >> b[1] >> b[0] >> b[3] >> b[2];
    if (!is || b[0] < 0 || b[1] >= kHistBins || b[2] < 0 || b[3] >= kHistBins || b[0] > b[1] || b[2] > b[3]) {
      set_error("remd_histogram_read: bad header in " + path);
      return REMD_ERR_IO;
    }
    std::fill(hist.begin(), hist.end(), 0);
    std::fill(ave.begin(), ave.end(), 0.0);
    for (int v = b[0]; v <= b[1]; v++)
      for (int p = b[2]; p <= b[3]; p++) {
        const size_t bin = (size_t)v * kHistBins + p;
        int n = 0;
        is >> dummy >> dummy >> n;
        hist[bin] = n;
        b[4] += n;
        for (int x = 0; x < kNumAvg; x++) {
          double a = 0.0;
          is >> a;
          ave[bin * kNumAvg + x] = a * (double)n;   // Histogram::SetAve
        }
      }
    if (!is) { set_error("remd_histogram_read: truncated " + path); return REMD_ERR_IO; }
    CK(cudaMemcpy(H.hist + nb * c, hist.data(), nb * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(H.ave + nb * kNumAvg * c, ave.data(), nb * kNumAvg * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(H.bounds + 5 * c, b, 5 * sizeof(int), cudaMemcpyHostToDevice));
  }
  return REMD_OK;
}

}  // extern "C"

namespace remd {
remd_status engine_create_carry(remd_handle from, const remd_system_desc* systems, int nens,
                                const int* reps_per_ens, const remd_replica_init* reps, const int* src_rep,
                                const int* src_ens, const int* grids, const unsigned long long* seeds,
                                const long long* steps, remd_precision prec, int device, cudaMemPool_t mempool,
                                remd_handle* out) {
  if (!src_rep || !src_ens || !grids || !seeds || !steps) {
    set_error("engine_create_carry: null argument");
    return REMD_ERR_INVALID;
  }
  if (from && ((from->prec == kF64) != (prec == REMD_PREC_FP64) || from->device != device)) {
    set_error("engine_create_carry: the previous handle has another precision or device");
    return REMD_ERR_INVALID;
  }
  Carry cy{from, src_rep, src_ens, grids, seeds, steps, mempool};
  return create_impl(systems, nens, reps_per_ens, reps, prec, device, &cy, out);
}
}  // namespace remd
