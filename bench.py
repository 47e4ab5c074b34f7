#!/usr/bin/env python
"""Benchmark: molecule-steps per second of the REMD hot path on one B200.

Workload (default): the 256-replica uneven batch -- 8 seeded ensembles, nmol
log-uniform in 64..2048, TIP3P/TIP4P/TIP5P, bulk / nanotube / nano-slit, rcut
8.5..12 A (remd_b200.systems.config4) -- with interval = 100 MD steps.  One
bench "step" is one REMD interval of the whole batch: 100 MD steps of every
replica (integrator, forces, wall), the interval start/end kernels and the
Metropolis T/P exchange of every ensemble, captured as one CUDA graph.

  value      whole-job mol-steps/s with the state resident in HBM, timed with
             CUDA events on the engine's stream (sum over the K intervals), L2
             flushed (256 MiB write) between intervals;
  e2e        the same metric through the public C-ABI call a user makes per
             interval: remd_execute_steps(T, P) from host arrays (H2D of the
             conditions, D2H of the 19 averages per replica) followed by the
             host-side Metropolis exchange of every ensemble;
  roofline   the force kernel (dominant): algorithmic FLOPs per launch
             (unordered pairs within rcut x 326 for TIP3P/TIP4P, x 515 for
             TIP5P) / its mean CUDA-event duration, against the measured FP32
             FMA peak of this GPU;
  cpu_baseline  the reference's own CPU code (oracle/_ref, generic FP64 build,
             replica-parallel on all host cores) on a bounded sample.

`--impl reference` times only that CPU baseline on the same workload and
prints its line.  Multi-GPU (`--gpus N` under torchrun): every rank runs its
own seeded copy of the workload (replicas only, no data-path collective),
value = total mol-steps / max over ranks of the device time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "mol-steps/s"
FLOP_PER_PAIR = {3: 326, 4: 326, 5: 515}


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--config", type=int, default=4, choices=[1, 2, 3, 4, 5])
    ap.add_argument("--jobs", type=int, default=8, help="config 5: jobs of the serving stream")
    ap.add_argument("--budget-gib", type=float, default=24.0, help="config 5: server HBM budget")
    ap.add_argument("--interval", type=int, default=100)
    ap.add_argument("--tile", type=int, default=0, help="force tile (0: autotuned)")
    ap.add_argument("--skin", type=float, default=0.0, help="neighbour skin in A (0: autotuned)")
    ap.add_argument("--seed", type=int, default=None, help="workload seed (default: the config index)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--no-serving", action="store_true",
                    help="config 4: skip the bounded serving sample (config 5's first --jobs jobs)")
    ap.add_argument("--cpu-steps", type=int, default=0, help="MD steps of the CPU sample (0: auto)")
    ap.add_argument("--study", choices=["drift", "lists", "clusters", "atomics"], default=None,
                    help="drift: NP Hamiltonian drift of the precision-study system (config 3), "
                         "FP32 form on every replica and FP64 vs FP32 on a subset")
    ap.add_argument("--drift-ps", type=float, default=100.0, help="drift study length (ps)")
    ap.add_argument("--drift-subset", type=int, default=8, help="replicas run in both forms")
    ap.add_argument("--drift-ref-ps", type=float, default=0.4,
                    help="drift study: window of the reference CPU FP64 leg (ps; 0 = skip)")
    ap.add_argument("--drift-ref-replicas", type=int, default=4,
                    help="drift study: replicas of the reference CPU FP64 leg")
    ap.add_argument("--equil-rounds", type=int, default=10,
                    help="untimed relaxation rounds of 20 steps + init_scaling")
    a = ap.parse_args(argv)
    if a.seed is None:
        a.seed = a.config
    return a


def workload(config, seed, interval):
    from remd_b200 import systems as S
    if config == 5:
        return [S.config5_job(seed, k, interval=interval)[0] for k in range(8)]
    if config == 4:
        return S.config4(seed=seed, interval=interval)
    fn = {1: S.config1, 2: S.config2, 3: S.config3}[config]
    ens = fn(seed=seed)
    for e in ens:
        e.spec.interval = interval
    return ens


def rank_workload(args, rank):
    """Replicas only: every rank runs its own seeded copy of the workload."""
    return workload(args.config, args.seed + 1000 * rank, args.interval)


def workload_desc(config, ens, interval):
    n = [e.spec.nmol for e in ens for _ in e.states]
    name = {4: "uneven batch: 8 ensembles / 256 replicas, TIP3P/4P/5P, bulk+tube+slit",
            1: "TIP4P nanotube N=128, 16 replicas", 2: "TIP4P slit N=512, 64 replicas",
            3: "TIP5P bulk N=1728, 128 replicas",
            5: "serving stream: the first 8 jobs' replicas"}[config]
    return {"workload": name, "config_index": config, "replicas": len(n),
            "molecules": int(sum(n)), "nmol_range": [int(min(n)), int(max(n))],
            "interval_steps": interval, "ensembles": len(ens),
            "models": sorted({e.spec.moltype.name for e in ens}),
            "l2": "flushed (256 MiB write) between timed intervals",
            "parallelism": "replicas-only"}


# ------------------------------------------------------------------ distributed
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return rank, world, local


def _reduce(x, world, op):
    """All-reduce one scalar (host plumbing for the bench line, not a data-path
    collective): on the current CUDA device under NCCL, on the host under gloo."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def reduce_max(x, world):
    import torch.distributed as dist
    return _reduce(x, world, dist.ReduceOp.MAX)


def reduce_sum(x, world):
    import torch.distributed as dist
    return _reduce(x, world, dist.ReduceOp.SUM)


def aggregate(local_ms, local_units, world):
    """Whole-job throughput of the replicas-only run: every rank's units over the
    slowest rank's device time.  Returns (value, max_ms, total_units)."""
    max_ms = reduce_max(local_ms, world)
    total = reduce_sum(local_units, world)
    return total / (max_ms * 1e-3), max_ms, total


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ------------------------------------------------------------------ clocks
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(gpu), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = [l.split(",") for l in open(self.f.name).read().splitlines() if l.strip()]
        os.unlink(self.f.name)
        sm, smax, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
                power.append(float(r[3]))
                for k, nm in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        load = [s for s in sm if s > 0.3 * max(sm)]
        return {"sm_mhz": float(np.median(load or sm)), "sm_max_mhz": float(max(smax)),
                "reasons": sorted(reasons), "samples": len(sm),
                "power_w_max": float(max(power)) if power else None}


# ------------------------------------------------------------------ CPU baseline (reference)
def cpu_baseline(ens, nsteps, nthreads, variant="generic"):
    """The reference's own CPU code (oracle/_ref; by default the generic FP64
    build, the one valid for every model and geometry), every replica advanced
    nsteps MD steps, replicas spread over nthreads host threads."""
    from oracle import oracle as O
    kind = "reference"
    if not O.reference_available(variant):
        if variant != "generic":
            return None
        kind = "port"
    refs = []
    t0 = time.perf_counter()
    for e in ens:
        for st in e.states:
            if kind == "reference":
                r = O.Reference(e.spec, st, e.spec.moltype_file, variant=variant)
                r.initialize_property()
            else:
                r = O.Oracle(e.spec, st)
                r.initialize_property()
            refs.append(r)
    setup = time.perf_counter() - t0
    molsteps = sum(e.spec.nmol for e in ens for _ in e.states) * nsteps
    t0 = time.perf_counter()
    if kind == "reference":
        O.reference_parallel_steps(refs, nsteps, nthreads)
        cores = nthreads
    else:
        for r in refs:
            r.steps(nsteps)
        cores = 1
    dt = time.perf_counter() - t0
    return {"value": molsteps / dt, "unit": METRIC, "cores": cores, "kind": kind, "cpu": cpu_model(),
            "sample": f"all {len(refs)} replicas x {nsteps} MD steps "
                      f"({'oracle/_ref ' + variant + ' build' if kind == 'reference' else 'C oracle'},"
                      f" replica-parallel over {cores} threads; {dt:.1f} s timed, setup {setup:.1f} s)",
            "seconds": dt}


def cpu_model():
    """The host CPU's model name and its logical CPU count (the affinity mask
    may allow fewer)."""
    name = "unknown"
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                name = ln.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return f"{name}, {os.cpu_count()} logical CPUs"


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def reference_arm(args, rank, world):
    if rank != 0:
        return
    ens = workload(args.config, args.seed, args.interval)
    from oracle import oracle as O
    nth = cpu_threads()
    total = sum(e.spec.nmol for e in ens for _ in e.states)
    # warm-up then K timed steps, each one MD step of every replica
    b = cpu_baseline(ens, max(args.warmup, 1), nth) if args.warmup > 0 else None
    res = cpu_baseline(ens, args.steps, nth)
    line = {"metric": METRIC, "value": res["value"], "unit": METRIC, "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": res["seconds"] * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_desc(args.config, ens, args.interval),
            "cpu_baseline": {k: res[k] for k in ("value", "unit", "cores", "kind", "cpu", "sample")},
            "e2e": {"value": res["value"], "unit": METRIC, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "note": "one step = one MD step of all replicas (bounded sample of the interval)"}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ serving (config 5)
def _gen_job(a):
    from remd_b200 import systems as S
    return S.config5_job(*a)


def make_jobs(seed, njobs):
    """The seeded job stream, generated on the host cores (spawned workers, so
    this is safe before or after CUDA is initialised)."""
    import multiprocessing as mp
    with mp.get_context("spawn").Pool(max(1, min(njobs, cpu_threads()))) as pool:
        return pool.map(_gen_job, [(seed, k) for k in range(njobs)])


def run_stream(jobs, arrivals, budget, dev, one_at_a_time, seed0=1000):
    """Feed the jobs to a server at their arrival times (host clock) and step it
    until all are done.  one_at_a_time: a job is submitted only when the server
    is empty (the plain one-job-at-a-time form).  Returns per-job latencies
    (arrival -> done, s), the makespan and the server's statistics."""
    from remd_b200 import engine as E
    srv = E.Server(budget_bytes=budget, device=dev)
    n = len(jobs)
    ids, done_t, state = [None] * n, [None] * n, [0] * n
    rounds = []   # (wall ms of one server round, molecule-steps of its interval)
    active = set()
    nxt = 0
    t0 = time.perf_counter()
    while True:
        now = time.perf_counter() - t0
        while nxt < n and arrivals[nxt] <= now and not (one_at_a_time and active):
            ens, nint = jobs[nxt]
            ids[nxt] = srv.submit(ens, nint, seed=seed0 + nxt)
            active.add(nxt)
            nxt += 1
        if not active:
            if nxt >= n:
                break
            time.sleep(max(arrivals[nxt] - now, 0.0))
            continue
        # the round's work: one interval of every job that is queued or running
        # (the server admits them all within the budget used here)
        units_round = sum(jobs[k][0].spec.nmol * jobs[k][0].nreplica * jobs[k][0].spec.interval
                          for k in active)
        changes0 = srv.stats()["batch_changes"]
        r0 = time.perf_counter()
        srv.step()
        rounds.append(((time.perf_counter() - r0) * 1e3, units_round,
                       srv.stats()["batch_changes"] != changes0))
        now = time.perf_counter() - t0
        for k in sorted(active):
            st = srv.poll(ids[k]).state
            if st >= 2:
                done_t[k], state[k] = now, st
                active.discard(k)
    stats = srv.stats()
    srv.close()
    lat = [done_t[k] - arrivals[k] for k in range(n)]
    ok = [k for k in range(n) if state[k] == 2]
    units = sum(jobs[k][0].spec.nmol * jobs[k][0].nreplica * jobs[k][0].spec.interval * jobs[k][1]
                for k in ok)
    span = max(done_t) - arrivals[0]
    return {"value": units / span, "makespan_s": span, "jobs_done": len(ok), "mol_steps": units,
            "p50_job_s": float(np.percentile(lat, 50)), "p99_job_s": float(np.percentile(lat, 99)),
            "p50_interval_ms": stats["p50_interval_ms"], "p99_interval_ms": stats["p99_interval_ms"],
            "intervals": stats["intervals_done"], "busy_s": stats["busy_s"],
            "batch_changes": stats["batch_changes"], "max_batch_change_ms": stats["max_batch_change_ms"],
            "max_graph_ms": stats["max_graph_ms"],
            # round time per million molecule-steps of its interval: the batch grows
            # and shrinks as jobs come and go, which alone spreads the round times
            "p50_round_ms_per_Mmolstep": float(np.percentile([r / (u * 1e-6) for r, u, _ in rounds], 50)),
            "p99_round_ms_per_Mmolstep": float(np.percentile([r / (u * 1e-6) for r, u, _ in rounds], 99)),
            # the same split by whether the round changed a batch (admission or exit)
            "rounds_steady": round_stats([x for x in rounds if not x[2]]),
            "rounds_with_batch_change": round_stats([x for x in rounds if x[2]])}


def round_stats(rounds):
    if not rounds:
        return {"n": 0}
    ms = [r for r, _, _ in rounds]
    per = [r / (u * 1e-6) for r, u, _ in rounds]
    return {"n": len(rounds), "p50_ms": float(np.percentile(ms, 50)), "p99_ms": float(np.percentile(ms, 99)),
            "p50_ms_per_Mmolstep": float(np.percentile(per, 50)),
            "p99_ms_per_Mmolstep": float(np.percentile(per, 99))}


def serving_sample(seed, njobs, warmup, budget_gib, dev, world):
    """The first `njobs` jobs of the seeded config-5 stream, served (continuous
    batching) and then one at a time, after `warmup` one-interval jobs."""
    from remd_b200 import systems as S
    jobs = make_jobs(seed, njobs)
    arrivals = S.config5_arrivals(seed, njobs)
    budget = int(budget_gib * (1 << 30))
    # warm-up: the first W jobs, one interval each (library load, context, graph capture)
    warm = [(e, 1) for e, _ in jobs[:max(warmup, 1)]]
    run_stream(warm, np.zeros(len(warm)), budget, dev, False, seed0=77)
    clocks = ClockSampler(dev)
    barrier(world)
    batched = run_stream(jobs, arrivals, budget, dev, False)
    barrier(world)
    clk = clocks.stop()
    single = run_stream(jobs, arrivals, budget, dev, True)
    return jobs, warm, batched, single, clk


def serving_arm(args, rank, world, local):
    import torch
    from remd_b200 import systems as S
    dev = local
    njobs = args.jobs
    torch.cuda.set_device(dev)
    jobs, warm, batched, single, clk = serving_sample(args.seed + 1000 * rank, njobs, args.warmup,
                                                      args.budget_gib, dev, world)
    value, max_s, total = aggregate(batched["makespan_s"] * 1e3, batched["mol_steps"], world)
    if rank == 0:
        n = [e.spec.nmol for e, _ in jobs]
        desc = {"workload": f"serving: Poisson stream, {S.SERVING_RATE:g} jobs/s, first {njobs} jobs; "
                            "nmol logU 96-4096, TIP3P/4P/5P, bulk+tube+slit, 8-64 replicas, "
                            "interval 100, ninterval 10-200",
                "config_index": 5, "jobs": njobs, "nmol_range": [min(n), max(n)],
                "replicas": int(sum(e.nreplica for e, _ in jobs)),
                "ninterval": [int(k) for _, k in jobs],
                "budget_gib": args.budget_gib, "parallelism": "replicas-only",
                "l2": "not flushed: a serving interval reads each job's state once per step "
                      "from its own buffers (working set of the batch > L2 for the larger jobs)"}
        line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
                "steps": njobs, "warmup": len(warm), "ms_per_step": max_s / njobs,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic", "config": desc,
                "latency": {k: batched[k] for k in ("p50_job_s", "p99_job_s", "p50_interval_ms",
                                                   "p99_interval_ms")},
                "served": batched, "one_at_a_time": single,
                "speedup_vs_one_at_a_time": batched["value"] / single["value"],
                "e2e": {"value": value, "unit": METRIC,
                        "note": "the server API is the host-facing call: job states are copied in "
                                "at admission and averages out every interval"},
                "clocks": clk}
        print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ precision study (config 3)
def _drift_run(eng, nint, dt_ps):
    """Advance `nint` intervals with fixed conditions (no exchange); H of every
    replica after each interval.  Returns (t_ns, H[nint, nrep])."""
    H = np.zeros((nint, eng.nrep))
    for k in range(nint):
        eng.execute_async()
        H[k] = eng.all_averages()[:, 11]
    t = (np.arange(nint) + 1) * dt_ps * 1e-3
    return t, H


def _drift_stats(t, H, nmol):
    """Per replica: least-squares slope of H(t) in kJ/mol per ns per molecule and
    the RMS residual about the line (kJ/mol per molecule)."""
    A = np.stack([t, np.ones_like(t)], axis=1)
    coef, *_ = np.linalg.lstsq(A, H, rcond=None)
    res = H - A @ coef
    rate = coef[0] / nmol
    return {"rate_median_abs": float(np.median(np.abs(rate))), "rate_max_abs": float(np.max(np.abs(rate))),
            "rate_mean": float(np.mean(rate)),
            "residual_rms_per_mol": float(np.sqrt(np.mean(res ** 2)) / nmol),
            "replicas": int(H.shape[1])}


def drift_study(args, rank, world, local):
    """NP Hamiltonian drift over `--drift-ps` of the precision-study system
    (TIP5P N=1728 bulk, rc 12 / rs 10, 128 replicas, 3-D barostat): every replica
    in the FP32 form, and `--drift-subset` replicas from the same equilibrated
    start in both the FP32 and the all-FP64 form.  Conditions are fixed (no
    exchange), so H = U + K + gkT ln s + Ps^2/2Q + Pv^2/2W + PV is conserved by
    the Nose-Poincare/Andersen equations up to the integrator's error."""
    import torch
    from remd_b200 import engine as E
    from remd_b200 import systems as S
    from remd_b200.inputs import ReplicaState
    if rank != 0:
        return
    dev = local
    torch.cuda.set_device(dev)
    ens = workload(3, args.seed, args.interval)
    e0 = ens[0]
    nmol = e0.spec.nmol
    dt_ps = e0.spec.dt * 1e-3 * args.interval
    nint = max(1, int(round(args.drift_ps / dt_ps)))
    eng = E.REMDGPU(ens, precision="fp32", device=dev)
    eng.equilibrate(rounds=args.equil_rounds, steps=20)
    sts = []
    for k in range(eng.nrep):
        g = eng.ConvertVariablesToHost(k)
        st0 = e0.states[k]
        sts.append(ReplicaState(g["r"], g["v"], g["q"], g["p"], st0.m, st0.I, g["s"], g["Ps"], g["Q"],
                                g["Pv"], g["W"], g["L"], g["T"], g["P"]))
    t0 = time.perf_counter()
    t, H32 = _drift_run(eng, nint, dt_ps)
    wall32 = time.perf_counter() - t0
    eng.close()
    sub = np.linspace(0, len(sts) - 1, args.drift_subset).round().astype(int)
    sub_states = [sts[k] for k in sub]
    one = S.Ensemble("drift", e0.spec, len(sub), 1, np.array([s.T for s in sub_states]),
                     np.array([s.P for s in sub_states]), sub_states)
    out = {}
    for prec in ("fp32", "fp64"):
        h = E.REMDGPU([one], precision=prec, device=dev)
        t0 = time.perf_counter()
        _, H = _drift_run(h, nint, dt_ps)
        out[prec] = (H, time.perf_counter() - t0)
        h.close()
    # the reference's own FP64 CPU build (oracle/_ref, generic switched path,
    # replica-parallel) from the first starts of the subset over a shorter
    # window, beside the engine's FP64 and FP32 forms over the same window
    ref_leg = None
    if args.drift_ref_ps > 0:
        from oracle import oracle as O
        if O.reference_available():
            samp = 10   # MD steps between H samples
            dts = e0.spec.dt * 1e-3 * samp
            nref = min(args.drift_ref_replicas, len(sub_states))
            nint_r = max(3, int(round(args.drift_ref_ps / dts)))
            starts = sub_states[:nref]
            tr = (np.arange(nint_r) + 1) * dts * 1e-3
            refs = [O.Reference(e0.spec, st, e0.spec.moltype_file) for st in starts]
            for r in refs:
                r.initialize_property()
            Hr = np.zeros((nint_r, nref))
            t0 = time.perf_counter()
            for k in range(nint_r):
                O.reference_parallel_steps(refs, samp, os.cpu_count() or 1)
                Hr[k] = [r.average()[11] for r in refs]
            wall_r = time.perf_counter() - t0
            short = S.Ensemble("drift_ref", e0.spec, nref, 1, np.array([s_.T for s_ in starts]),
                               np.array([s_.P for s_ in starts]), starts)
            eng_short = {}
            for prec in ("fp64", "fp32"):
                h = E.REMDGPU([short], precision=prec, device=dev, interval=samp)
                _, H = _drift_run(h, nint_r, dts)
                eng_short[prec] = _drift_stats(tr, H, nmol)
                h.close()
            ref_leg = {"duration_ps": nint_r * dts, "samples": nint_r, "sample_steps": samp,
                       "reference_cpu_fp64": dict(_drift_stats(tr, Hr, nmol), wall_s=wall_r,
                                                  threads=os.cpu_count(),
                                                  build="oracle/_ref generic FP64 (-DSWITCHING)"),
                       "engine_fp64": eng_short["fp64"], "engine_fp32": eng_short["fp32"]}
    line = {"metric": "NP Hamiltonian drift", "unit": "kJ/mol per ns per molecule",
            "value": _drift_stats(t, H32, nmol)["rate_median_abs"], "higher_is_better": False,
            "study": "drift", "duration_ps": nint * dt_ps, "intervals": nint,
            "config": {"workload": "TIP5P bulk N=1728, rc 12 / rs 10, 128 replicas, 3-D barostat, "
                                   "fixed conditions (no exchange)", "config_index": 3,
                       "equilibration": f"{args.equil_rounds} x (20 steps + init_scaling)"},
            "fp32_all": dict(_drift_stats(t, H32, nmol), wall_s=wall32),
            "subset": [int(k) for k in sub],
            "fp32_subset": dict(_drift_stats(t, out["fp32"][0], nmol), wall_s=out["fp32"][1]),
            "fp64_subset": dict(_drift_stats(t, out["fp64"][0], nmol), wall_s=out["fp64"][1]),
            "short_window_vs_reference_cpu": ref_leg,
            "data": "synthetic"}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ force step per system (list builds)
def lists_study(args, rank, world, local):
    """Force-step time per launch (CUDA events over 50 MD steps, list rebuilds
    included: remd_profile_split) at fixed tile 32 and several skins, for the config-4
    batch and for the largest systems of the serving stream (N = 4096: a 50 A
    TIP5P bulk box, a 1.4 um TIP4P nanotube, a 115 A TIP3P slit; 8 replicas
    each), with a hash of the positions and momenta after one more interval
    (the trajectory does not depend on how the lists are built)."""
    import ctypes
    import hashlib

    import torch
    from remd_b200 import engine as E
    from remd_b200 import systems as S
    if rank != 0:
        return
    torch.cuda.set_device(local)
    out = {}

    def measure(name, ens, skin, nsteps):
        eng = E.REMDGPU(ens, precision="fp32", device=local, interval=10)
        eng.set_tuning(32, skin)
        eng.execute_nsteps(20)
        prof = (ctypes.c_double * 5)()
        E._check(E.lib().remd_profile_split(eng.h, nsteps, prof))
        eng.ExecuteSteps(np.concatenate([e.T for e in ens]), np.concatenate([e.P for e in ens]))
        h = hashlib.sha1()
        for r in range(min(eng.nrep, 8)):
            g = eng.ConvertVariablesToHost(r)
            h.update(g["r"].tobytes())
            h.update(g["p"].tobytes())
        out[name] = {"force_ms": prof[1] + prof[2] + prof[3], "integrate_ms": prof[0], "head_ms": prof[1],
                     "lists_ms": prof[2], "pairs_ms": prof[3], "rebuilt_replicas_per_step": prof[4],
                     "skin": skin, "tile": 32, "trajectory_sha1": h.hexdigest()}
        eng.close()

    c4 = S.config4(seed=4)
    for skin in (0.2, 0.6, 1.0):
        measure(f"config4_skin{skin}", c4, skin, 50)
    for model, confined, wall, rc in [("tip5p", 0, 0.0, 12.0), ("tip4p", 1, 7.0, 10.0), ("tip3p", 2, 12.0, 11.0)]:
        e = S.make_ensemble("big", model, confined, 4096, wall, rc, rc - 1.0, 4, 2, 250, 350, 0.1e6, 0.1e6, 41)
        for skin in (0.2, 1.0):
            measure(f"n4096_{model}_confined{confined}_skin{skin}", [e], skin, 30)
    print(json.dumps({"study": "lists", "unit": "ms per MD step", "systems": out}), flush=True)


# ------------------------------------------------------------------ Newton's third law by cluster pairs (host)
def _morton3(c):
    """Z-order code of non-negative integer cell coordinates (n x 3, < 2^10)."""
    code = np.zeros(len(c), dtype=np.int64)
    for bit in range(10):
        for d in range(3):
            code |= ((c[:, d] >> bit) & 1).astype(np.int64) << (3 * bit + d)
    return code


def clusters_study(args, rank, world, local):
    """How much pair work a Newton's-third-law scheme over spatial clusters of M
    molecules would evaluate, against the engine's exact full lists, on the
    config-4 systems (replica 0 of every ensemble, the seeded liquid-density
    start).  Molecules are ordered along a Z-order curve of ~3.1 A cells and cut
    into clusters of M consecutive molecules; a pair of clusters is evaluated
    when their bounding boxes come within rcut (minimum image), every molecule
    pair of it (M^2, or M(M-1)/2 on the diagonal) once.  The full lists evaluate
    every pair within rcut twice (2U).  Host-only (numpy)."""
    if rank != 0:
        return
    ens = workload(4, args.seed, args.interval)
    out = {}
    tot = {}
    for e in ens:
        st = e.states[0]
        L = np.asarray(st.L, float)
        x = (np.asarray(st.r, float) % 1.0) * L
        n = len(x)
        rc = e.spec.rcut
        d = x[:, None, :] - x[None, :, :]
        d -= L * np.round(d / L)
        r2 = (d ** 2).sum(-1)
        U = int(((r2 < rc * rc).sum() - n) // 2)
        cell = np.floor(x / 3.1).astype(np.int64)
        order = np.argsort(_morton3(cell), kind="stable")
        row = {"nmol": n, "rcut": rc, "confined": e.spec.confined, "pairs_within_rc": U}
        for M in (4, 8, 16, 32):
            ids = [order[k:k + M] for k in range(0, n, M)]
            cen, half = [], []
            for c in ids:
                p = x[c]
                q = p - L * np.round((p - p[0]) / L)   # unwrap around the first member
                lo, hi = q.min(0), q.max(0)
                cen.append(0.5 * (lo + hi))
                half.append(0.5 * (hi - lo))
            cen, half = np.array(cen), np.array(half)
            dc = cen[:, None, :] - cen[None, :, :]
            dc -= L * np.round(dc / L)
            gap = np.maximum(np.abs(dc) - (half[:, None, :] + half[None, :, :]), 0.0)
            near = (gap ** 2).sum(-1) < rc * rc
            sizes = np.array([len(c) for c in ids])
            iu = np.triu_indices(len(ids), 1)
            slots = int((sizes[iu[0]] * sizes[iu[1]])[near[iu]].sum() + (sizes * (sizes - 1) // 2).sum())
            row[f"M{M}"] = {"slots": slots, "in_range_fraction": U / slots, "work_vs_full_lists": slots / (2 * U)}
            t = tot.setdefault(M, [0, 0])
            t[0] += slots
            t[1] += 2 * U
        out[e.name] = row
    summary = {f"M{M}": {"work_vs_full_lists": s_ / u2, "in_range_fraction": u2 / 2 / s_}
               for M, (s_, u2) in tot.items()}
    print(json.dumps({"study": "clusters", "workload": "config 4, replica 0 of each ensemble (seeded start)",
                      "summary": summary, "ensembles": out}), flush=True)


def atomics_study(args, rank, world, local):
    """Integer-add throughput (remd_measure_atomics) beside the pair work a
    Newton's-third-law force step would add with it: config 4's unordered pairs
    within rcut (seed 4, the bench's equilibrated state has 7.96 M) x 7 values
    (force, space-frame torque and its scalar part) per pair."""
    import ctypes

    from remd_b200 import engine as E
    rates = (ctypes.c_double * 4)()
    E._check(E.lib().remd_measure_atomics(local, rates))
    names = ["shared_u64", "shared_u32", "cluster_peer_u64", "global_u64"]
    adds = 7.96e6 * 7
    print(json.dumps({"study": "atomics", "unit": "G adds/s",
                      "rates": {n: rates[k] for k, n in enumerate(names)},
                      "adds_per_force_step": adds,
                      "us_per_force_step_at_rate": {n: adds / (rates[k] * 1e9) * 1e6
                                                    for k, n in enumerate(names)}}), flush=True)


# ------------------------------------------------------------------ engine arm
def profile_traffic():
    """DRAM bytes per force launch from the committed ncu summary, if present."""
    p = os.path.join(ROOT, "profiles", "force_kernel_config4.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.strip().startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


def force_accuracy(eng, ens, dev):
    """FP32 forces of the bench's own (equilibrated, advanced) configurations
    against the FP64 form of the engine on the same snapshots (the FP64 form is
    pinned to the FP64 oracle by the parity tests).  Per replica: force and
    torque RMS relative error (||F32 - F64||_2 / ||F64||_2 over all molecules),
    potential-energy and virial relative error; reported as the max over
    replicas."""
    from remd_b200 import engine as E
    from remd_b200.inputs import ReplicaState
    eng.compute_forces()
    sts, got = [], []
    k = 0
    for e in ens:
        for st0 in e.states:
            g = eng.ConvertVariablesToHost(k)
            sts.append(ReplicaState(g["r"], g["v"], g["q"], g["p"], st0.m, st0.I, g["s"], g["Ps"],
                                    g["Q"], g["Pv"], g["W"], g["L"], g["T"], g["P"]))
            got.append(g)
            k += 1
    ref = E.REMDGPU(ens, precision="fp64", device=dev, states=sts)
    ref.compute_forces()
    fe, ne, ue, ve = [], [], [], []
    worst = None
    meta = [(ei, e.spec.moltype.name, e.spec.confined, round(e.spec.rcut, 3), e.spec.nmol)
            for ei, e in enumerate(ens) for _ in e.states]
    for k, g in enumerate(got):
        h = ref.ConvertVariablesToHost(k)
        fe.append(np.linalg.norm(g["f"] - h["f"]) / np.linalg.norm(h["f"]))
        ne.append(np.linalg.norm(g["n"] - h["n"]) / np.linalg.norm(h["n"]))
        ue.append(abs(g["pot"] - h["pot"]) / abs(h["pot"]))
        ve.append(np.linalg.norm(g["vir"] - h["vir"]) / np.linalg.norm(h["vir"]))
        if worst is None or fe[-1] > worst[0]:
            dm = np.linalg.norm(g["f"] - h["f"], axis=1)
            i = int(np.argmax(dm))
            worst = (fe[-1], {"replica": k, "ensemble": meta[k][0], "model": meta[k][1],
                              "confined": meta[k][2], "rcut": meta[k][3], "nmol": meta[k][4],
                              "box": [float(x) for x in h["L"]], "molecule": i,
                              "abs_err": float(dm[i]),
                              "force_abs": float(np.linalg.norm(h["f"][i])),
                              "force_abs_median": float(np.median(np.linalg.norm(h["f"], axis=1)))})
    ref.close()
    return {"reference": "FP64 form of this engine on the same snapshots",
            "replicas": len(got),
            "force_rms_rel_max": float(max(fe)), "force_rms_rel_median": float(np.median(fe)),
            "torque_rms_rel_max": float(max(ne)),
            "pot_rel_max": float(max(ue)), "pot_rel_median": float(np.median(ue)),
            "virial_rel_max": float(max(ve)),
            "replicas_over_force_gate": int(sum(1 for x in fe if x > 1e-5)),
            "worst": worst[1],
            "gates": {"force_rms_rel": 1e-5, "pot_rel": 1e-6}}


def engine_arm(args, rank, world, local):
    import ctypes

    import torch

    from remd_b200 import engine as E
    dev = local
    torch.cuda.set_device(dev)
    ens = rank_workload(args, rank)
    eng = E.REMDGPU(ens, precision="fp32", device=dev)
    if args.tile or args.skin:
        eng.set_tuning(args.tile or 64, args.skin or 1.0)
    T = np.concatenate([e.T for e in ens])
    P = np.concatenate([e.P for e in ens])
    nmol_total = int(sum(e.spec.nmol for e in ens for _ in e.states))
    mol_steps_per_interval = nmol_total * args.interval
    stream = torch.cuda.ExternalStream(E.lib().remd_stream(eng.h))
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{dev}")
    # untimed: relax the lattice start (init_scaling every 20 steps), then warm up
    eng.equilibrate(rounds=args.equil_rounds, steps=20)
    # untimed: the autotuner picks (tile, skin) on this batch; the trajectory does
    # not depend on the choice
    if args.tile or args.skin:
        tuning = {"tile": args.tile or 64, "skin": args.skin or 1.0, "autotuned": False}
    else:
        # 100 steps per trial: each trial starts with a list build, which a shorter
        # window over-weights (it favours the largest skin)
        t, k, tms = eng.autotune(nsteps=100)
        tuning = {"tile": t, "skin": k, "autotuned": True, "ms_per_md_step": tms}
    # one bench step = one REMD interval: `interval` MD steps of every replica and
    # the Metropolis exchange of every ensemble, all on the device
    eng.enable_device_exchange([(e.ntemp, e.npress) for e in ens], seed=2024 + rank)
    for _ in range(args.warmup):
        eng.execute_async(T, P)
    eng.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    clocks = ClockSampler(dev)
    barrier(world)
    torch.cuda.synchronize()
    eng.synchronize()
    w0 = time.perf_counter()
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(float(k))
        evs[k][0].record(stream)
        eng.execute_async()
        evs[k][1].record(stream)
    eng.synchronize()
    torch.cuda.synchronize()
    barrier(world)
    wall = time.perf_counter() - w0
    clk = clocks.stop()
    ms = [a.elapsed_time(b) for a, b in evs]
    local_ms = float(sum(ms))
    value, max_ms, total_units = aggregate(local_ms, mol_steps_per_interval * args.steps, world)
    statuses = [eng.replica_status(r) for r in range(eng.nrep)]
    launches = eng.launches_per_interval() * args.steps   # with the device exchange, as timed

    # roofline of the force kernel: per-launch algorithmic FLOPs / event duration
    eng.compute_forces()
    flops = 0.0
    pairs = 0
    k = 0
    for e in ens:
        for _ in e.states:
            pr = int(E.lib().remd_replica_pair_count(eng.h, k))
            pairs += pr
            flops += pr * FLOP_PER_PAIR[e.spec.moltype.nsite]
            k += 1
    prof = (ctypes.c_double * 2)()
    E._check(E.lib().remd_profile_steps(eng.h, 50, prof))   # 50 steps: list rebuilds at their usual rate
    force_ms, integ_ms = prof[1], prof[0]
    peak = ctypes.c_double()
    E._check(E.lib().remd_measure_fp32_peak(dev, ctypes.byref(peak)))
    achieved = flops / (force_ms * 1e-3) / 1e12
    roof = {"bound": "fp32",
            "kernel": "force step: k_replica_head (PsPv + D4, list decision, cell sort) + "
                      "k_force_lists (list rebuild, pairs within rcut) + "
                      "k_force_pairs (pair forces, wall, A2M)",
            "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
            "frac": achieved / peak.value,
            "peak_source": "measured: register-resident FP32 FMA chains on all SMs "
                           "(remd_measure_fp32_peak); MEASURED_PEAKS.json has no FP32 figure",
            "traffic": profile_traffic(), "pairs_per_launch": pairs,
            "flops_per_launch": flops, "force_ms": force_ms, "integrate_ms": integ_ms,
            "timing": "force_ms: CUDA events around the force launches of 50 MD steps run one "
                      "launch chain at a time (remd_profile_steps, rebuilds included)"}
    # the same FLOPs over the MD step of the timed schedule (the interval graph's
    # concurrent chains; the step also holds the integrate and head kernels)
    step_ms = (max_ms / args.steps) / args.interval
    roof["in_timed_schedule"] = {"ms_per_md_step": step_ms, "achieved": flops / (step_ms * 1e-3) / 1e12,
                                 "frac": flops / (step_ms * 1e-3) / 1e12 / peak.value}

    acc = None if args.no_accuracy else force_accuracy(eng, ens, dev)

    # end to end through the public C-ABI call (host buffers, host exchange)
    e2e = None
    eng.enable_device_exchange(None)
    if not args.no_e2e:
        grids = [(e.ntemp, e.npress) for e in ens]
        idx = [np.arange(e.nreplica, dtype=np.int32) for e in ens]
        Ts = [e.T.copy() for e in ens]
        Ps = [e.P.copy() for e in ens]
        rng = np.random.default_rng(123 + rank)
        off = np.cumsum([0] + [e.nreplica for e in ens])

        def interval(step):
            eng.ExecuteSteps(np.concatenate(Ts), np.concatenate(Ps))
            avg = eng.all_averages()
            for i, e in enumerate(ens):
                a = avg[off[i]:off[i + 1]]
                E.exchange_host(grids[i][0], grids[i][1], e.spec.pconstant, step, idx[i], Ts[i],
                                Ps[i], a[:, 0] + a[:, 1] + a[:, 2], a[:, 3],
                                rng.random(max(e.nreplica // 2, 1)))
        # untimed: the first call re-instantiates the interval graph (without the
        # device exchange that the device-timed loop used)
        interval(0)
        barrier(world)
        t0 = time.perf_counter()
        for step in range(args.steps):
            interval(step + 1)
        e2e_s = reduce_max(time.perf_counter() - t0, world)
        e2e = {"value": total_units / e2e_s, "unit": METRIC,
               "h2d_bytes_per_step": int(2 * 8 * eng.nrep),
               "d2h_bytes_per_step": int(19 * 8 * eng.nrep),
               "path": "remd_execute_steps(T,P) + remd_get_all_averages + remd_exchange_host per ensemble"}

    # plain per-replica FP64 form on a sample (one replica of every ensemble)
    plain = None
    if not args.no_plain and rank == 0:
        psteps = 10
        tot_ms, tot_units = 0.0, 0
        for e in ens:
            st = e.states[0]
            from remd_b200 import systems as S
            one = E.REMDGPU([S.Ensemble("p", e.spec, 1, 1, e.T[:1], e.P[:1], [st])],
                            precision="fp64", device=dev, interval=psteps)
            s1 = torch.cuda.ExternalStream(E.lib().remd_stream(one.h))
            one.execute_async(e.T[:1], e.P[:1])
            one.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(s1)
            one.execute_async()
            b.record(s1)
            one.synchronize()
            tot_ms += a.elapsed_time(b)
            tot_units += e.spec.nmol * psteps
            one.close()
        plain = {"value": tot_units / (tot_ms * 1e-3), "unit": METRIC, "dtype": "f64",
                 "sample": f"one replica of each of the {len(ens)} ensembles, alone, "
                           f"{psteps} steps each (one launch sequence per replica)"}

    # a bounded sample of the serving stream (config 5), beside the batch
    serving = None
    if not args.no_serving and args.config == 4 and rank == 0 and world == 1:
        jobs, _, sb, s1, _ = serving_sample(5, args.jobs, 1, args.budget_gib, dev, 1)
        serving = {"workload": f"config 5: the first {len(jobs)} jobs of the seeded Poisson stream "
                               f"(nmol {min(e.spec.nmol for e, _ in jobs)}-"
                               f"{max(e.spec.nmol for e, _ in jobs)}, "
                               f"{sum(e.nreplica for e, _ in jobs)} replicas)",
                   "served_mol_steps_per_s": sb["value"], "one_at_a_time_mol_steps_per_s": s1["value"],
                   "speedup_vs_one_at_a_time": sb["value"] / s1["value"],
                   "p50_interval_ms": sb["p50_interval_ms"], "p99_interval_ms": sb["p99_interval_ms"],
                   "p50_job_s": sb["p50_job_s"], "p99_job_s": sb["p99_job_s"],
                   "intervals": sb["intervals"], "jobs_done": sb["jobs_done"],
                   "batch_changes": sb["batch_changes"], "max_batch_change_ms": sb["max_batch_change_ms"],
                   "max_graph_ms": sb["max_graph_ms"],
                   "p50_round_ms_per_Mmolstep": sb["p50_round_ms_per_Mmolstep"],
                   "p99_round_ms_per_Mmolstep": sb["p99_round_ms_per_Mmolstep"],
                   "rounds_steady": sb["rounds_steady"],
                   "rounds_with_batch_change": sb["rounds_with_batch_change"],
                   "interval_latency": "wall time of one server round: admission, any batch change, "
                                       "the interval's graph launch and the averages' read-back"}

    cpu = None
    if not args.no_cpu_baseline and rank == 0 and world == 1:
        nst = args.cpu_steps or 2
        cpu = cpu_baseline(ens, nst, cpu_threads())
        cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "cpu", "sample")}
        # config 1 (TIP4P nanotube) is the one workload the reference's tuned 4-site
        # CPU path is valid for: also time it as shipped (makefile.gnu flags, FP32
        # forces, replicas one after another) and as the tuned FP64 build
        if args.config == 1:
            forms = {}
            for name, variant, threads in [("shipped_fp32_4site_serial", "shipped", 1),
                                           ("tuned_fp64_4site_replica_parallel", "tuned4", cpu_threads())]:
                r = cpu_baseline(ens, max(nst, 200), threads, variant)
                if r:
                    forms[name] = {k: r[k] for k in ("value", "unit", "cores", "sample")}
            cpu["other_reference_forms"] = forms

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": dict(workload_desc(args.config, ens, args.interval), tuning=tuning),
                "gpu_launches": launches,
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
                "latency": {"p50_interval_ms": float(np.percentile(ms, 50)),
                            "p99_interval_ms": float(np.percentile(ms, 99)),
                            "samples": len(ms)},
                "accuracy": acc,
                "serving": serving,
                "plain_fp64": plain,
                "speedup_vs_plain_fp64": (value / world / plain["value"]) if plain else None,
                "wall_s": wall, "interval_ms": [round(x, 3) for x in ms],
                "replica_status_nonzero": int(sum(1 for s in statuses if s))}
        print(json.dumps(line), flush=True)
    eng.close()


def main():
    args = parse_args()
    rank, world, local = dist_setup(args)
    try:
        if args.impl == "reference":
            reference_arm(args, rank, world)
        elif args.study == "drift":
            drift_study(args, rank, world, local)
        elif args.study == "lists":
            lists_study(args, rank, world, local)
        elif args.study == "clusters":
            clusters_study(args, rank, world, local)
        elif args.study == "atomics":
            atomics_study(args, rank, world, local)
        elif args.config == 5:
            serving_arm(args, rank, world, local)
        else:
            engine_arm(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
