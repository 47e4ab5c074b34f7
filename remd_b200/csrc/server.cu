// server.cu -- continuous batching of REMD jobs on one GPU.
//
// A job is one REMD system (an ensemble: ntemp x npress replicas) to be run for
// `ninterval` intervals (MD + Metropolis exchange each).  remd_server_step()
// is one scheduling round:
//   1. cancelled jobs leave the batch, freeing their HBM budget;
//   2. queued jobs are admitted in arrival order while their estimated device
//      footprint fits the budget (and their interval matches the batch's);
//   3. if the batch changed, a new engine handle is built for the new set: the
//      jobs that keep running are copied into it from the previous handle on
//      the device (molecule state, scalars and H0, pending conditions,
//      exchange index, counter and seed), only new jobs' states come from the
//      host; the handle's arrays come from a memory pool the server keeps, and
//      its interval graph is the previous one updated in place;
//   4. every job in the batch advances one interval in one graph launch.
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
#include <mutex>
#include <string>
#include <vector>

#include "../../include/remd_b200.h"
#include "hostio.h"

namespace remd {
remd_status engine_get_exchange(remd_handle h, long long* steps, int* index);
size_t engine_bytes(remd_handle h);
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

struct remd_server_s {
  std::mutex mu;
  size_t budget = 0;
  int device = 0;
  remd_precision prec = REMD_PREC_FP32;
  remd_job_id next_id = 1;
  std::vector<Job*> jobs;          // every job ever submitted (owned)
  std::vector<Job*> queue;         // waiting, in arrival order
  std::vector<Job*> active;        // in the current batch, in batch order
  remd_handle batch = nullptr;
  cudaMemPool_t mempool = nullptr; // every batch handle's arrays (kept between batch changes)
  bool dirty = false;
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
static remd_status read_index(remd_server_s* S) {
  if (!S->batch) return REMD_OK;
  int total = 0;
  for (Job* j : S->active) total += j->nrep();   // every active job is in the batch here
  std::vector<long long> steps(S->active.size());
  std::vector<int> idx(total);
  remd_status st = engine_get_exchange(S->batch, steps.data(), idx.data());
  if (st != REMD_OK) return st;
  for (Job* j : S->active) {
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

// A batch handle for the active jobs, continuing the previous one's.  On
// failure the previous handle is left as it was.
static remd_status build_batch(remd_server_s* S) {
  if (S->active.empty()) {
    if (S->batch) { remd_destroy(S->batch); S->batch = nullptr; }
    return REMD_OK;
  }
  std::vector<remd_system_desc> sys;
  std::vector<int> per, grids, src_rep, src_ens;
  std::vector<remd_replica_init> init;
  std::vector<unsigned long long> seeds;
  std::vector<long long> steps;
  for (Job* j : S->active) {
    sys.push_back(j->sys);
    per.push_back(j->nrep());
    grids.push_back(j->nt);
    grids.push_back(j->np);
    seeds.push_back(j->seed);
    steps.push_back(j->step);
    src_ens.push_back(S->batch ? j->ens_in_batch : -1);
    for (int k = 0; k < j->nrep(); k++) {
      remd_replica_init ri{};
      if (S->batch && j->ens_in_batch >= 0) {
        src_rep.push_back(j->rep_in_batch + k);
      } else {
        src_rep.push_back(-1);
        fill_init(j->reps[k], ri);
      }
      init.push_back(ri);
    }
  }
  remd_handle nb = nullptr;
  remd_status st = engine_create_carry(S->batch, sys.data(), (int)sys.size(), per.data(), init.data(),
                                       src_rep.data(), src_ens.data(), grids.data(), seeds.data(), steps.data(),
                                       S->prec, S->device, S->mempool, &nb);
  if (st != REMD_OK) return st;
  if (S->batch) remd_destroy(S->batch);
  S->batch = nb;
  int rep = 0;
  for (size_t e = 0; e < S->active.size(); e++) {
    Job* j = S->active[e];
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
  if (S->batch) remd_destroy(S->batch);
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

remd_status remd_server_step(remd_server S, int* pending) {
  if (!S) return REMD_ERR_INVALID;
  std::lock_guard<std::mutex> lk(S->mu);
  const double t_round = now_s();
  // 1. leave: cancelled jobs (finished ones left at the end of their last round)
  for (size_t e = 0; e < S->active.size();) {
    Job* j = S->active[e];
    if (j->state == 4) {
      S->dirty = true;
      S->in_use -= j->bytes;
      j->t_end = now_s() - S->t0;
      S->active.erase(S->active.begin() + e);
    } else {
      e++;
    }
  }
  // 2. admit in arrival order while the budget allows
  while (!S->queue.empty()) {
    Job* j = S->queue.front();
    if (!S->active.empty() && j->sys.interval != S->active[0]->sys.interval) break;
    if (S->in_use + j->bytes > S->budget) break;
    S->queue.erase(S->queue.begin());
    S->active.push_back(j);
    S->in_use += j->bytes;
    j->state = 1;
    j->t_start = now_s() - S->t0;
    S->dirty = true;
  }
  // 3. a new batch handle if the membership changed
  if (S->dirty) {
    const double tb = now_s();
    remd_status st = build_batch(S);
    if (st != REMD_OK && st != REMD_ERR_CUDA) {
      // a job whose own state cannot start (e.g. a neighbour list over capacity
      // in the initial force call) fails alone: find it by building each job
      // that has not run yet on its own, then build again without the failures
      bool any = false;
      for (size_t e = 0; e < S->active.size();) {
        Job* j = S->active[e];
        const remd_status sj = j->ens_in_batch < 0 ? job_alone_status(S, j) : REMD_OK;
        if (sj != REMD_OK) {
          j->state = 3;
          j->status = sj;
          j->t_end = now_s() - S->t0;
          S->in_use -= j->bytes;
          S->active.erase(S->active.begin() + e);
          any = true;
        } else {
          e++;
        }
      }
      if (any) st = build_batch(S);
    }
    if (st != REMD_OK) {
      for (Job* j : S->active) { j->state = 3; j->status = st; j->t_end = now_s() - S->t0; }
      S->active.clear();
      S->in_use = 0;
      S->dirty = false;
      if (S->batch) { remd_destroy(S->batch); S->batch = nullptr; }
      return st;
    }
    S->dirty = false;
    S->batch_changes++;
    S->max_change_ms = std::max(S->max_change_ms, (now_s() - tb) * 1e3);
  }
  // 4. one interval (MD + exchange) for every running job
  if (S->batch) {
    const double t0 = now_s();
    remd_status st = remd_execute_steps_device(S->batch);
    S->busy_s += now_s() - t0;
    S->max_graph_ms = std::max(S->max_graph_ms, engine_last_graph_ms(S->batch));
    S->intervals_done++;
    int total = 0;
    for (Job* j : S->active) total += j->nrep();
    // A replica that went non-finite or overflowed its neighbour list fails its
    // own job only: the replicas of the other jobs are independent of it, their
    // interval is complete and valid, and they keep running.
    std::vector<char> bad(S->active.size(), 0);
    if (st == REMD_ERR_NONFINITE || st == REMD_ERR_NEIGHBOR_OVERFLOW) {
      int nbad = 0;
      for (size_t e = 0; e < S->active.size(); e++)
        for (int k = 0; k < S->active[e]->nrep(); k++) {
          int w = 0;
          if (remd_replica_status(S->batch, S->active[e]->rep_in_batch + k, &w) != REMD_OK) w = 1;
          if (w != 0 && !bad[e]) { bad[e] = 1; nbad++; }
        }
      if (nbad > 0) {
        for (size_t e = 0; e < S->active.size(); e++)
          if (bad[e]) { S->active[e]->state = 3; S->active[e]->status = st; }
        st = REMD_OK;
      }
    }
    std::vector<double> avg((size_t)total * 19);
    if (st == REMD_OK) st = remd_get_all_averages(S->batch, avg.data());
    int rep = 0;
    bool left = false;
    for (size_t e = 0; e < S->active.size(); e++) {
      Job* j = S->active[e];
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
      remd_status pst = read_index(S);   // the leaving jobs' final condition index
      if (pst != REMD_OK) return pst;
      for (size_t e = 0; e < S->active.size();) {
        Job* j = S->active[e];
        if (j->state == 2 || j->state == 3) {
          j->t_end = now_s() - S->t0;
          if (j->state == 2) { S->job_s.push_back(j->t_end - j->t_submit); S->jobs_done++; }
          S->in_use -= j->bytes;
          S->active.erase(S->active.begin() + e);
          S->dirty = true;
        } else {
          e++;
        }
      }
    }
    // the latency of the whole round: admission, any batch change and the interval
    S->interval_ms.push_back((now_s() - t_round) * 1e3);
    if (st != REMD_OK) return st;
  }
  if (pending) *pending = (int)(S->queue.size() + S->active.size());
  return REMD_OK;
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
