// server.cu -- continuous batching of REMD jobs on one GPU.
//
// A job is one REMD system (an ensemble: ntemp x npress replicas) to be run for
// `ninterval` intervals (MD + Metropolis exchange each).  remd_server_step()
// is one scheduling round:
//   1. cancelled jobs leave the batch, freeing their HBM budget;
//   2. queued jobs are admitted in arrival order while their estimated device
//      footprint fits the budget, each into the batch of its MD interval length
//      (jobs of different lengths run as separate batches, side by side);
//   3. if the batch changed, a new engine handle is built for the new set: the
//      jobs that keep running are copied into it from the previous handle on
//      the device (molecule state, scalars and H0, pending conditions,
//      exchange index, counter and seed), only new jobs' states come from the
//      host; the handle's arrays come from a memory pool the server keeps, and
//      its interval graph is the previous one updated in place;
//   4. every job advances one interval: one graph launch per batch, the batches'
//      graphs running at the same time on their own streams.
// Forces are a pure function of the positions (see pair_loop_f32) and every
// per-replica reduction has a fixed order, so a job's trajectory is the same
// bit for bit whether it runs alone or with any batch mates, and across batch
// changes (tests/test_gpu_server.py).  A replica that goes non-finite or
// overflows its neighbour list fails its own job only.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <future>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/remd_b200.h"
#include "hostio.h"

namespace remd {
remd_status engine_get_exchange(remd_handle h, long long* steps, int* index);
size_t engine_bytes(remd_handle h);
void engine_prepare_wall(const remd_system_desc& s);
double engine_last_graph_ms(remd_handle h);
remd_status engine_create_carry(remd_handle from, const remd_system_desc* systems, int nens,
                                const int* reps_per_ens, const remd_replica_init* reps, const int* src_rep,
                                const int* src_ens, const int* grids, const unsigned long long* seeds,
                                const long long* steps, remd_precision prec, int device, cudaMemPool_t mempool,
                                remd_handle* out);
}  // namespace remd

using namespace remd;

namespace {

// A replica's initial state, kept on the host from submission until the job
// first joins a batch (afterwards its state lives on the device).
struct Rep {
  std::vector<double> r, v, q, p, m, I;
  double s, Ps, Q, Pv[3], W, L[3], T, P;
};

struct Job {
  remd_job_id id;
  remd_system_desc sys;
  int nt, np;
  int ninterval, done = 0;
  unsigned long long seed;
  int state = 0;   // 0 queued, 1 running, 2 done, 3 failed, 4 cancelled
  remd_status status = REMD_OK;
  double t_submit = 0, t_start = 0, t_end = 0;
  std::vector<Rep> reps;
  std::vector<int> index;          // condition slot -> replica (read back when the job leaves)
  long long step = 0;              // next exchange list type = step % 4
  int ens_in_batch = -1;           // ensemble of the current batch handle, -1 before admission
  int rep_in_batch = -1;           // its first replica there
  std::vector<double> avg;         // latest averages, nrep x 19
  std::future<void> wall;          // its wall table, computed in the background from submission
  size_t bytes = 0;
  int nrep() const { return nt * np; }
};

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// Device footprint of a job, with the engine's own layout formula.
size_t estimate_bytes(const remd_system_desc& s, int nrep) {
  const double rl = s.rcut + 1.0;
  int cap = ((int)std::ceil(0.1 * 4.0 / 3.0 * M_PI * rl * rl * rl) + 7) / 8 * 8;
  cap = std::min(cap, s.nmol - 1);
  const size_t ntile = (s.nmol + 127) / 128;
  // skin list + FP32 per-step list: 2 x 2 bytes per slot
  const size_t per_rep = (size_t)s.nmol * (176 + 80 + 16 + 4) + ntile * (size_t)cap * 128 * 4 +
                         ntile * (3 * 8 + 64 + 64 + 16) + 1024;
  return per_rep * nrep + (size_t)std::max(s.nfwall, 0) * 16 + 4096;
}

double pct(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double x = q * (v.size() - 1);
  const size_t i = (size_t)x;
  const double f = x - i;
  return i + 1 < v.size() ? v[i] * (1 - f) + v[i + 1] * f : v[i];
}

}  // namespace

// The running jobs that share one MD interval length: one engine handle (one
// interval graph) advances all of them by one interval per round.
struct Batch {
  int interval = 0;
  std::vector<Job*> active;        // in batch order
  remd_handle h = nullptr;
  bool dirty = false;              // membership changed since h was built
};

struct remd_server_s {
  std::mutex mu;
  size_t budget = 0;
  int device = 0;
  remd_precision prec = REMD_PREC_FP32;
  remd_job_id next_id = 1;
  std::vector<Job*> jobs;          // every job ever submitted (owned)
  std::vector<Job*> queue;         // waiting, in arrival order
  std::vector<Batch> batches;      // running jobs, one batch per MD interval length
  cudaMemPool_t mempool = nullptr; // every batch handle's arrays (kept between batch changes)
  size_t in_use = 0;
  double t0 = now_s();
  std::vector<double> interval_ms, job_s;
  long long jobs_done = 0, intervals_done = 0, mol_steps = 0;
  double busy_s = 0.0;
  long long batch_changes = 0;
  double max_change_ms = 0.0, max_graph_ms = 0.0;

  Job* find(remd_job_id id) {
    for (Job* j : jobs)
      if (j->id == id) return j;
    return nullptr;
  }
};

// The exchange index and interval counter of every job in the batch (a few
// bytes per replica): read before a job leaves, for its result.
static remd_status read_index(Batch& B) {
  if (!B.h) return REMD_OK;
  int total = 0;
  for (Job* j : B.active) total += j->nrep();   // every active job is in the handle here
  std::vector<long long> steps(B.active.size());
  std::vector<int> idx(total);
  remd_status st = engine_get_exchange(B.h, steps.data(), idx.data());
  if (st != REMD_OK) return st;
  for (Job* j : B.active) {
    j->step = steps[j->ens_in_batch];
    j->index.assign(idx.begin() + j->rep_in_batch, idx.begin() + j->rep_in_batch + j->nrep());
  }
  return REMD_OK;
}

static void fill_init(const Rep& R, remd_replica_init& ri) {
  ri.r = R.r.data(); ri.v = R.v.data(); ri.q = R.q.data(); ri.p = R.p.data();
  ri.mass = R.m.data(); ri.inertia = R.I.data();
  ri.s = R.s; ri.Ps = R.Ps; ri.Q = R.Q; ri.W = R.W; ri.T = R.T; ri.P = R.P;
  for (int x = 0; x < 3; x++) { ri.Pv[x] = R.Pv[x]; ri.L[x] = R.L[x]; }
}

// A batch handle for the batch's active jobs, continuing its previous one.  On
// failure the previous handle is left as it was.
static remd_status build_batch(remd_server_s* S, Batch& B) {
  if (B.active.empty()) {
    if (B.h) { remd_destroy(B.h); B.h = nullptr; }
    return REMD_OK;
  }
  std::vector<remd_system_desc> sys;
  std::vector<int> per, grids, src_rep, src_ens;
  std::vector<remd_replica_init> init;
  std::vector<unsigned long long> seeds;
  std::vector<long long> steps;
  for (Job* j : B.active) {
    sys.push_back(j->sys);
    per.push_back(j->nrep());
    grids.push_back(j->nt);
    grids.push_back(j->np);
    seeds.push_back(j->seed);
    steps.push_back(j->step);
    src_ens.push_back(B.h ? j->ens_in_batch : -1);
    for (int k = 0; k < j->nrep(); k++) {
      remd_replica_init ri{};
      if (B.h && j->ens_in_batch >= 0) {
        src_rep.push_back(j->rep_in_batch + k);
      } else {
        src_rep.push_back(-1);
        fill_init(j->reps[k], ri);
      }
      init.push_back(ri);
    }
  }
  remd_handle nb = nullptr;
  remd_status st = engine_create_carry(B.h, sys.data(), (int)sys.size(), per.data(), init.data(),
                                       src_rep.data(), src_ens.data(), grids.data(), seeds.data(), steps.data(),
                                       S->prec, S->device, S->mempool, &nb);
  if (st != REMD_OK) return st;
  if (B.h) remd_destroy(B.h);
  B.h = nb;
  int rep = 0;
  for (size_t e = 0; e < B.active.size(); e++) {
    Job* j = B.active[e];
    j->ens_in_batch = (int)e;
    j->rep_in_batch = rep;
    rep += j->nrep();
    std::vector<Rep>().swap(j->reps);   // its state lives on the device now
  }
  return REMD_OK;
}

// The status of building job j alone (its initial force call and H0).
static remd_status job_alone_status(remd_server_s* S, Job* j) {
  std::vector<remd_replica_init> init(j->nrep());
  for (int k = 0; k < j->nrep(); k++) fill_init(j->reps[k], init[k]);
  const int per = j->nrep();
  remd_handle h = nullptr;
  const remd_status st = remd_create(&j->sys, 1, &per, init.data(), S->prec, S->device, &h);
  if (h) remd_destroy(h);
  return st;
}

extern "C" {

remd_status remd_server_open(size_t hbm_budget_bytes, int device, remd_precision prec,
                             remd_server* out) {
  if (!out || hbm_budget_bytes == 0) {
    set_error("remd_server_open: need an output handle and a budget > 0");
    return REMD_ERR_INVALID;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
    set_error("no CUDA device");
    return REMD_ERR_NO_DEVICE;
  }
  if (cudaSetDevice(device) != cudaSuccess) {
    set_error("remd_server_open: bad device");
    return REMD_ERR_INVALID;
  }
  // the batch handles' arrays: a pool that keeps what it has reserved, so that
  // a batch change allocates without going back to the driver
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  cudaMemPool_t pool = nullptr;
  if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
    cudaGetLastError();
    set_error("remd_server_open: cannot create the device memory pool");
    return REMD_ERR_CUDA;
  }
  unsigned long long keep = ~0ull;
  cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  auto* S = new remd_server_s;
  S->budget = hbm_budget_bytes;
  S->device = device;
  S->prec = prec;
  S->mempool = pool;
  *out = S;
  return REMD_OK;
}

remd_status remd_server_close(remd_server S) {
  if (!S) return REMD_OK;
  for (Batch& B : S->batches)
    if (B.h) remd_destroy(B.h);
  if (S->mempool) {
    cudaDeviceSynchronize();
    cudaMemPoolDestroy(S->mempool);
  }
  for (Job* j : S->jobs) delete j;
  delete S;
  return REMD_OK;
}

remd_status remd_job_submit(remd_server S, const remd_job_desc* jd, remd_job_id* id) {
  if (!S || !jd || !id || !jd->reps || jd->ntemp < 1 || jd->npress < 1 || jd->ninterval < 1 ||
      jd->system.nmol < 2) {
    set_error("remd_job_submit: bad job description");
    return REMD_ERR_INVALID;
  }
  auto* j = new Job;
  j->sys = jd->system;
  j->nt = jd->ntemp;
  j->np = jd->npress;
  j->ninterval = jd->ninterval;
  j->seed = jd->seed;
  const int n = jd->system.nmol;
  for (int k = 0; k < j->nrep(); k++) {
    const remd_replica_init& ri = jd->reps[k];
    if (!ri.r || !ri.v || !ri.q || !ri.p || !ri.mass || !ri.inertia) {
      delete j;
      set_error("remd_job_submit: null state array");
      return REMD_ERR_INVALID;
    }
    Rep R;
    R.r.assign(ri.r, ri.r + 3 * n); R.v.assign(ri.v, ri.v + 3 * n);
    R.q.assign(ri.q, ri.q + 4 * n); R.p.assign(ri.p, ri.p + 4 * n);
    R.m.assign(ri.mass, ri.mass + n); R.I.assign(ri.inertia, ri.inertia + 3 * n);
    R.s = ri.s; R.Ps = ri.Ps; R.Q = ri.Q; R.W = ri.W; R.T = ri.T; R.P = ri.P;
    for (int x = 0; x < 3; x++) { R.Pv[x] = ri.Pv[x]; R.L[x] = ri.L[x]; }
    j->reps.push_back(R);
    j->index.push_back(k);
  }
  j->bytes = estimate_bytes(j->sys, j->nrep());
  std::lock_guard<std::mutex> lk(S->mu);
  if (j->bytes > S->budget) {
    delete j;
    set_error("remd_job_submit: the job alone exceeds the HBM budget");
    return REMD_ERR_OOM;
  }
  // a confined job's wall table (about a second of host time for a 65536-entry
  // tube table on few cores) is computed while the job waits in the queue, so
  // that admitting it does not stall the round that builds its batch; without a
  // thread for it, the batch build computes it
  if (j->sys.confined > 0) {
    try {
      j->wall = std::async(std::launch::async, engine_prepare_wall, j->sys);
    } catch (...) {
    }
  }
  j->id = S->next_id++;
  j->t_submit = now_s() - S->t0;
  S->jobs.push_back(j);
  S->queue.push_back(j);
  *id = j->id;
  return REMD_OK;
}

remd_status remd_job_poll(remd_server S, remd_job_id id, remd_job_info* info) {
  if (!S || !info) return REMD_ERR_INVALID;
  std::lock_guard<std::mutex> lk(S->mu);
  Job* j = S->find(id);
  if (!j) { set_error("unknown job"); return REMD_ERR_INVALID; }
  info->state = j->state;
  info->intervals_done = j->done;
  info->submit_s = j->t_submit;
  info->start_s = j->t_start;
  info->end_s = j->t_end;
  info->status = j->status;
  return REMD_OK;
}

remd_status remd_job_cancel(remd_server S, remd_job_id id) {
  if (!S) return REMD_ERR_INVALID;
  std::lock_guard<std::mutex> lk(S->mu);
  Job* j = S->find(id);
  if (!j) { set_error("unknown job"); return REMD_ERR_INVALID; }
  if (j->state == 0) {
    S->queue.erase(std::find(S->queue.begin(), S->queue.end(), j));
    j->state = 4;
    j->status = REMD_ERR_CANCELLED;
    j->t_end = now_s() - S->t0;
  } else if (j->state == 1) {
    j->state = 4;   // leaves the batch at the next scheduling round
    j->status = REMD_ERR_CANCELLED;
  }
  return REMD_OK;
}

remd_status remd_job_result(remd_server S, remd_job_id id, double* averages, int* index) {
  if (!S) return REMD_ERR_INVALID;
  std::lock_guard<std::mutex> lk(S->mu);
  Job* j = S->find(id);
  if (!j) { set_error("unknown job"); return REMD_ERR_INVALID; }
  if (j->state != 2) { set_error("job not finished"); return REMD_ERR_INVALID; }
  if (averages) std::memcpy(averages, j->avg.data(), j->avg.size() * 8);
  if (index) std::memcpy(index, j->index.data(), j->index.size() * 4);
  return REMD_OK;
}

// Builds the handle of a batch whose membership changed.  A job whose own
// state cannot start (e.g. a neighbour list over capacity in the initial force
// call) fails alone: it is found by building each job of the batch that has not
// run yet on its own, and the batch is built again without the failures.
static remd_status rebuild(remd_server_s* S, Batch& B) {
  const double tb = now_s();
  remd_status st = build_batch(S, B);
  if (st != REMD_OK && st != REMD_ERR_CUDA) {
    bool any = false;
    for (size_t e = 0; e < B.active.size();) {
      Job* j = B.active[e];
      const remd_status sj = j->ens_in_batch < 0 ? job_alone_status(S, j) : REMD_OK;
      if (sj != REMD_OK) {
        j->state = 3;
        j->status = sj;
        j->t_end = now_s() - S->t0;
        S->in_use -= j->bytes;
        B.active.erase(B.active.begin() + e);
        any = true;
      } else {
        e++;
      }
    }
    if (any) st = build_batch(S, B);
  }
  if (st != REMD_OK) {
    for (Job* j : B.active) {
      j->state = 3;
      j->status = st;
      j->t_end = now_s() - S->t0;
      S->in_use -= j->bytes;
    }
    B.active.clear();
    if (B.h) { remd_destroy(B.h); B.h = nullptr; }
  }
  B.dirty = false;
  S->batch_changes++;
  S->max_change_ms = std::max(S->max_change_ms, (now_s() - tb) * 1e3);
  return st;
}

// After an interval of batch B: the averages of every job, failures local to a
// job, finished jobs leaving.  st is the interval's status.
static remd_status collect(remd_server_s* S, Batch& B, remd_status st) {
  int total = 0;
  for (Job* j : B.active) total += j->nrep();
  // A replica that went non-finite or overflowed its neighbour list fails its
  // own job only: the replicas of the other jobs are independent of it, their
  // interval is complete and valid, and they keep running.
  std::vector<char> bad(B.active.size(), 0);
  if (st == REMD_ERR_NONFINITE || st == REMD_ERR_NEIGHBOR_OVERFLOW) {
    int nbad = 0;
    for (size_t e = 0; e < B.active.size(); e++)
      for (int k = 0; k < B.active[e]->nrep(); k++) {
        int w = 0;
        if (remd_replica_status(B.h, B.active[e]->rep_in_batch + k, &w) != REMD_OK) w = 1;
        if (w != 0 && !bad[e]) { bad[e] = 1; nbad++; }
      }
    if (nbad > 0) {
      for (size_t e = 0; e < B.active.size(); e++)
        if (bad[e]) { B.active[e]->state = 3; B.active[e]->status = st; }
      st = REMD_OK;
    }
  }
  std::vector<double> avg((size_t)total * 19);
  if (st == REMD_OK) st = remd_get_all_averages(B.h, avg.data());
  int rep = 0;
  bool left = false;
  for (size_t e = 0; e < B.active.size(); e++) {
    Job* j = B.active[e];
    j->avg.assign(avg.begin() + (size_t)rep * 19, avg.begin() + (size_t)(rep + j->nrep()) * 19);
    rep += j->nrep();
    if (bad[e]) { left = true; continue; }
    if (st != REMD_OK) { j->state = 3; j->status = st; left = true; continue; }
    j->done++;
    S->mol_steps += (long long)j->sys.nmol * j->nrep() * j->sys.interval;
    if (j->done >= j->ninterval) {
      j->state = 2;
      left = true;
    }
  }
  if (left) {
    remd_status pst = read_index(B);   // the leaving jobs' final condition index
    if (pst != REMD_OK) return pst;
    for (size_t e = 0; e < B.active.size();) {
      Job* j = B.active[e];
      if (j->state == 2 || j->state == 3) {
        j->t_end = now_s() - S->t0;
        if (j->state == 2) { S->job_s.push_back(j->t_end - j->t_submit); S->jobs_done++; }
        S->in_use -= j->bytes;
        B.active.erase(B.active.begin() + e);
        B.dirty = true;
      } else {
        e++;
      }
    }
  }
  return st;
}

remd_status remd_server_step(remd_server S, int* pending) {
  if (!S) return REMD_ERR_INVALID;
  std::lock_guard<std::mutex> lk(S->mu);
  const double t_round = now_s();
  // 1. leave: cancelled jobs (finished ones left at the end of their last round)
  for (Batch& B : S->batches)
    for (size_t e = 0; e < B.active.size();) {
      Job* j = B.active[e];
      if (j->state == 4) {
        B.dirty = true;
        S->in_use -= j->bytes;
        j->t_end = now_s() - S->t0;
        B.active.erase(B.active.begin() + e);
      } else {
        e++;
      }
    }
  // 2. admit in arrival order while the budget allows, each job into the batch
  //    of its MD interval length
  while (!S->queue.empty()) {
    Job* j = S->queue.front();
    if (S->in_use + j->bytes > S->budget) break;
    S->queue.erase(S->queue.begin());
    if (j->wall.valid()) j->wall.get();   // its wall table is in the engine's cache
    Batch* B = nullptr;
    for (Batch& b : S->batches)
      if (b.interval == j->sys.interval) B = &b;
    if (!B) {
      S->batches.emplace_back();
      B = &S->batches.back();
      B->interval = j->sys.interval;
    }
    B->active.push_back(j);
    B->dirty = true;
    S->in_use += j->bytes;
    j->state = 1;
    j->t_start = now_s() - S->t0;
  }
  // 3. new handles for the batches whose membership changed
  remd_status first_err = REMD_OK;
  for (Batch& B : S->batches)
    if (B.dirty) {
      const remd_status st = rebuild(S, B);
      if (st != REMD_OK && first_err == REMD_OK) first_err = st;
    }
  // 4. one interval (MD + exchange) of every running job: the batches' graphs
  //    are launched first, so that they run at the same time on their streams
  bool ran = false;
  std::vector<remd_status> launched(S->batches.size(), REMD_OK);
  const double t0 = now_s();
  for (size_t b = 0; b < S->batches.size(); b++)
    if (S->batches[b].h) launched[b] = remd_execute_steps_async(S->batches[b].h, nullptr, nullptr);
  for (size_t b = 0; b < S->batches.size(); b++) {
    Batch& B = S->batches[b];
    if (!B.h) continue;
    remd_status st = launched[b];
    if (st == REMD_OK) st = remd_synchronize(B.h);
    S->max_graph_ms = std::max(S->max_graph_ms, engine_last_graph_ms(B.h));
    ran = true;
    st = collect(S, B, st);
    if (st != REMD_OK && first_err == REMD_OK) first_err = st;
  }
  if (ran) {
    S->busy_s += now_s() - t0;
    S->intervals_done++;
    // the latency of the whole round: admission, any batch change and the interval
    S->interval_ms.push_back((now_s() - t_round) * 1e3);
  }
  // batches left without jobs release their handles
  for (size_t b = 0; b < S->batches.size();) {
    Batch& B = S->batches[b];
    if (B.active.empty()) {
      if (B.h) remd_destroy(B.h);
      S->batches.erase(S->batches.begin() + b);
    } else {
      b++;
    }
  }
  size_t running = 0;
  for (const Batch& B : S->batches) running += B.active.size();
  if (pending) *pending = (int)(S->queue.size() + running);
  return first_err;
}

remd_status remd_job_bytes(const remd_job_desc* jd, size_t* out) {
  if (!jd || !out || jd->ntemp < 1 || jd->npress < 1 || jd->system.nmol < 2) return REMD_ERR_INVALID;
  *out = estimate_bytes(jd->system, jd->ntemp * jd->npress);
  return REMD_OK;
}

remd_status remd_server_stats_get(remd_server S, remd_server_stats* o) {
  if (!S || !o) return REMD_ERR_INVALID;
  std::lock_guard<std::mutex> lk(S->mu);
  o->jobs_done = S->jobs_done;
  o->intervals_done = S->intervals_done;
  o->mol_steps = S->mol_steps;
  o->p50_interval_ms = pct(S->interval_ms, 0.50);
  o->p99_interval_ms = pct(S->interval_ms, 0.99);
  o->p50_job_s = pct(S->job_s, 0.50);
  o->p99_job_s = pct(S->job_s, 0.99);
  o->busy_s = S->busy_s;
  o->bytes_in_use = (long long)S->in_use;
  o->budget_bytes = (long long)S->budget;
  o->batch_changes = S->batch_changes;
  o->max_batch_change_ms = S->max_change_ms;
  o->max_graph_ms = S->max_graph_ms;
  return REMD_OK;
}

}  // extern "C"
