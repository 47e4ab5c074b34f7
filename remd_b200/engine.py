"""Python mirror of the reference's REMDGPU call surface (src/remdgpu.h:92-238)
over the C-ABI of libremd_b200.so (include/remd_b200.h).

    eng = REMDGPU(ensembles, precision="fp32")
    eng.ExecuteSteps(T, P)          # one interval for every replica
    avg = eng.GetAverages(rep)      # the 19 Average fields
    st  = eng.ConvertVariablesToHost(rep)

The compute path is the CUDA library; there is no CPU fallback.  If the library
is missing it is built with nvcc (remd_b200/csrc/Makefile); if that fails, or
no GPU is visible, the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from .inputs import ReplicaState

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libremd_b200.so")
NUM_AVG = 19
AVG_NAMES = ["LJ", "CLMB", "WALL", "VOL", "TRA", "ROT", "T", "P", "Px", "Py", "Pz",
             "TOT", "DRF", "TSTs", "TSTv", "BSTx", "BSTy", "BSTz", "DUMMY"]
STATUS = {0: "OK", 1: "INVALID", 2: "OOM", 3: "TIMEOUT", 4: "NONFINITE", 5: "CANCELLED",
          6: "CUDA", 7: "IO", 8: "NEIGHBOR_OVERFLOW", 9: "NO_DEVICE", 10: "RANGE"}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class RemdError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"remd status {STATUS.get(status, status)}: {msg}")
        self.status = status


class SystemDesc(C.Structure):
    _fields_ = [("nmol", C.c_int), ("nsite", C.c_int), ("site_r", (C.c_double * 3) * 5),
                ("site_mass", C.c_double * 5), ("site_sigma", C.c_double * 5),
                ("site_eps", C.c_double * 5), ("site_charge", C.c_double * 5),
                ("tconstant", C.c_int), ("pconstant", C.c_int), ("confined", C.c_int),
                ("dt_fs", C.c_double), ("rcut", C.c_double), ("rswitch", C.c_double),
                ("nfwall", C.c_int), ("wall_length", C.c_double), ("sgm_wall", C.c_double),
                ("eps_wall", C.c_double), ("rho_wall", C.c_double), ("interval", C.c_int)]


class ReplicaInit(C.Structure):
    _fields_ = [("r", _dp), ("v", _dp), ("q", _dp), ("p", _dp), ("mass", _dp),
                ("inertia", _dp), ("s", C.c_double), ("Ps", C.c_double), ("Q", C.c_double),
                ("Pv", C.c_double * 3), ("W", C.c_double), ("L", C.c_double * 3),
                ("T", C.c_double), ("P", C.c_double)]


class StateView(C.Structure):
    _fields_ = [("r", _dp), ("v", _dp), ("q", _dp), ("p", _dp), ("f", _dp), ("n", _dp),
                ("s", C.c_double), ("Ps", C.c_double), ("Q", C.c_double),
                ("Pv", C.c_double * 3), ("W", C.c_double), ("L", C.c_double * 3),
                ("T", C.c_double), ("P", C.c_double), ("H0", C.c_double),
                ("pot", C.c_double), ("lj", C.c_double), ("clmb", C.c_double),
                ("wall", C.c_double), ("vir", C.c_double * 3)]


_LIB = None


def build_library():
    subprocess.run(["make", "-s", "-C", os.path.join(HERE, "csrc")], check=True)


def lib():
    """Load libremd_b200.so (building it first if it is absent)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            build_library()
        L = C.CDLL(LIB_PATH)
        L.remd_last_error.restype = C.c_char_p
        L.remd_version.restype = C.c_char_p
        L.remd_last_pair_count.restype = C.c_longlong
        L.remd_create.argtypes = [C.POINTER(SystemDesc), C.c_int, _ip, C.POINTER(ReplicaInit),
                                  C.c_int, C.c_int, C.POINTER(C.c_void_p)]
        for fn in ["remd_destroy", "remd_compute_forces", "remd_synchronize",
                   "remd_execute_steps_device", "remd_num_replicas",
                   "remd_launches_per_interval", "remd_last_pair_count"]:
            getattr(L, fn).argtypes = [C.c_void_p]
        L.remd_execute_steps.argtypes = [C.c_void_p, _dp, _dp]
        L.remd_execute_nsteps.argtypes = [C.c_void_p, C.c_int]
        L.remd_rescale_velocities.argtypes = [C.c_void_p]
        L.remd_replica_pair_count.restype = C.c_longlong
        L.remd_replica_pair_count.argtypes = [C.c_void_p, C.c_int]
        L.remd_stream.restype = C.c_void_p
        L.remd_stream.argtypes = [C.c_void_p]
        L.remd_profile_steps.argtypes = [C.c_void_p, C.c_int, _dp]
        L.remd_profile_split.argtypes = [C.c_void_p, C.c_int, _dp]
        L.remd_measure_fp32_peak.argtypes = [C.c_int, _dp]
        L.remd_measure_atomics.argtypes = [C.c_int, _dp]
        L.remd_autotune.argtypes = [C.c_void_p, C.c_int, _ip, _dp, _dp]
        L.remd_execute_steps_async.argtypes = [C.c_void_p, _dp, _dp]
        L.remd_get_averages.argtypes = [C.c_void_p, C.c_int, _dp]
        L.remd_get_all_averages.argtypes = [C.c_void_p, _dp]
        L.remd_get_state.argtypes = [C.c_void_p, C.c_int, C.POINTER(StateView)]
        L.remd_replica_nmol.argtypes = [C.c_void_p, C.c_int]
        L.remd_replica_status.argtypes = [C.c_void_p, C.c_int, _ip]
        L.remd_set_tuning.argtypes = [C.c_void_p, C.c_int, C.c_double]
        L.remd_exchange_device.argtypes = [C.c_void_p, _ip, C.c_long, _dp, C.c_ulonglong]
        L.remd_get_conditions.argtypes = [C.c_void_p, _ip, _dp, _dp]
        L.remd_enable_device_exchange.argtypes = [C.c_void_p, _ip, C.c_ulonglong, C.c_longlong]
        L.remd_server_open.argtypes = [C.c_size_t, C.c_int, C.c_int, C.POINTER(C.c_void_p)]
        L.remd_server_close.argtypes = [C.c_void_p]
        L.remd_job_submit.argtypes = [C.c_void_p, C.POINTER(JobDesc), C.POINTER(C.c_longlong)]
        L.remd_job_poll.argtypes = [C.c_void_p, C.c_longlong, C.POINTER(JobInfo)]
        L.remd_job_cancel.argtypes = [C.c_void_p, C.c_longlong]
        L.remd_job_result.argtypes = [C.c_void_p, C.c_longlong, _dp, _ip]
        L.remd_server_step.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
        L.remd_server_stats_get.argtypes = [C.c_void_p, C.POINTER(ServerStats)]
        L.remd_job_bytes.argtypes = [C.POINTER(JobDesc), C.POINTER(C.c_size_t)]
        L.remd_force_snapshot_noalloc.argtypes = [C.POINTER(SystemDesc), C.c_void_p, C.c_void_p, _dp,
                                                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                  C.c_void_p]
        L.remd_write_chk.argtypes = [C.c_void_p, C.c_int, C.c_char_p]
        L.remd_write_gro.argtypes = [C.c_void_p, C.c_int, C.c_char_p, C.c_char_p,
                                     C.POINTER(C.c_char_p)]
        L.remd_wall_table.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                      C.c_double, _dp]
        L.remd_read_chk.argtypes = [C.c_char_p, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.remd_write_chk_arrays.argtypes = [C.c_char_p, C.c_int, C.c_int, _dp, _dp, _dp, _dp,
                                            C.c_double, _dp, _dp, _dp]
        L.remd_exchange_host.argtypes = [C.c_int, C.c_int, C.c_int, C.c_long, _ip, _dp, _dp,
                                         _dp, _dp, _dp, _ip, _ip]
        _LIB = L
    return _LIB


def _check(st):
    if st != 0:
        raise RemdError(st, lib().remd_last_error().decode())


def _p(a, t=_dp):
    return a.ctypes.data_as(t)


def system_desc(spec) -> SystemDesc:
    """remd_system_desc from a SystemSpec (moltype in moltype.txt units)."""
    d = SystemDesc()
    mt = spec.moltype
    d.nmol, d.nsite = spec.nmol, mt.nsite
    for k in range(mt.nsite):
        for x in range(3):
            d.site_r[k][x] = mt.r[k, x]
        d.site_mass[k], d.site_sigma[k] = mt.mass[k], mt.sigma[k]
        d.site_eps[k], d.site_charge[k] = mt.eps[k], mt.charge[k]
    d.tconstant, d.pconstant, d.confined = spec.tconstant, spec.pconstant, spec.confined
    d.dt_fs, d.rcut, d.rswitch = spec.dt, spec.rcut, spec.rswitch
    d.nfwall, d.wall_length = spec.nfwall, spec.wall_length
    d.sgm_wall, d.eps_wall, d.rho_wall = spec.sgm_wall, spec.eps_wall, spec.rho_wall
    d.interval = spec.interval
    return d


class JobDesc(C.Structure):
    _fields_ = [("system", SystemDesc), ("ntemp", C.c_int), ("npress", C.c_int),
                ("reps", C.POINTER(ReplicaInit)), ("ninterval", C.c_int), ("seed", C.c_ulonglong)]


class JobInfo(C.Structure):
    _fields_ = [("state", C.c_int), ("intervals_done", C.c_int), ("submit_s", C.c_double),
                ("start_s", C.c_double), ("end_s", C.c_double), ("status", C.c_int)]


class ServerStats(C.Structure):
    _fields_ = [("jobs_done", C.c_longlong), ("intervals_done", C.c_longlong),
                ("mol_steps", C.c_longlong), ("p50_interval_ms", C.c_double),
                ("p99_interval_ms", C.c_double), ("p50_job_s", C.c_double),
                ("p99_job_s", C.c_double), ("busy_s", C.c_double),
                ("bytes_in_use", C.c_longlong), ("budget_bytes", C.c_longlong),
                ("batch_changes", C.c_longlong), ("max_batch_change_ms", C.c_double),
                ("max_graph_ms", C.c_double)]


def _replica_inits(states):
    keep = []
    inits = (ReplicaInit * len(states))()
    for k, st in enumerate(states):
        arrs = [np.ascontiguousarray(getattr(st, f), dtype=np.float64)
                for f in ("r", "v", "q", "p", "m", "I")]
        keep.append(arrs)
        ri = inits[k]
        ri.r, ri.v, ri.q, ri.p, ri.mass, ri.inertia = [_p(a) for a in arrs]
        ri.s, ri.Ps, ri.Q, ri.W, ri.T, ri.P = st.s, st.Ps, st.Q, st.W, st.T, st.P
        for x in range(3):
            ri.Pv[x] = st.Pv[x]
            ri.L[x] = st.L[x]
    return inits, keep


class Server:
    """Continuous batching of REMD jobs (include/remd_b200.h, serving section)."""

    def __init__(self, budget_bytes, precision="fp32", device=0):
        self.h = C.c_void_p()
        _check(lib().remd_server_open(C.c_size_t(int(budget_bytes)), device,
                                      1 if precision == "fp64" else 0, C.byref(self.h)))

    @staticmethod
    def job_desc(ensemble, ninterval, seed=0, interval=None):
        d = JobDesc()
        d.system = system_desc(ensemble.spec)
        if interval is not None:
            d.system.interval = interval
        d.ntemp, d.npress = ensemble.ntemp, ensemble.npress
        inits, keep = _replica_inits(ensemble.states)
        d.reps = inits
        d.ninterval, d.seed = ninterval, seed
        return d, (inits, keep)

    @staticmethod
    def job_bytes(ensemble):
        d, keep = Server.job_desc(ensemble, 1)
        out = C.c_size_t()
        _check(lib().remd_job_bytes(C.byref(d), C.byref(out)))
        return out.value

    def submit(self, ensemble, ninterval, seed=0, interval=None):
        d = JobDesc()
        d.system = system_desc(ensemble.spec)
        if interval is not None:
            d.system.interval = interval
        d.ntemp, d.npress = ensemble.ntemp, ensemble.npress
        inits, keep = _replica_inits(ensemble.states)
        d.reps = inits
        d.ninterval, d.seed = ninterval, seed
        jid = C.c_longlong()
        _check(lib().remd_job_submit(self.h, C.byref(d), C.byref(jid)))
        return jid.value

    def step(self):
        pending = C.c_int()
        _check(lib().remd_server_step(self.h, C.byref(pending)))
        return pending.value

    def poll(self, jid):
        info = JobInfo()
        _check(lib().remd_job_poll(self.h, C.c_longlong(jid), C.byref(info)))
        return info

    def cancel(self, jid):
        _check(lib().remd_job_cancel(self.h, C.c_longlong(jid)))

    def result(self, jid, nrep):
        avg = np.zeros((nrep, NUM_AVG))
        idx = np.zeros(nrep, dtype=np.int32)
        _check(lib().remd_job_result(self.h, C.c_longlong(jid), _p(avg), _p(idx, _ip)))
        return avg, idx

    def stats(self):
        s = ServerStats()
        _check(lib().remd_server_stats_get(self.h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in ServerStats._fields_}

    def close(self):
        if self.h:
            lib().remd_server_close(self.h)
            self.h = C.c_void_p()


class REMDGPU:
    """All replicas of one or more ensembles on one GPU (src/remdgpu.h:92-238)."""

    def __init__(self, ensembles, precision="fp32", device=0, states=None, interval=None):
        L = lib()
        self.ensembles = list(ensembles)
        descs = []
        for e in self.ensembles:
            d = system_desc(e.spec)
            if interval is not None:
                d.interval = interval
            descs.append(d)
        n_e = len(descs)
        self.reps_per_ens = np.array([len(e.states) for e in self.ensembles], dtype=np.int32)
        states = states or [s for e in self.ensembles for s in e.states]
        self._keep = []
        inits = (ReplicaInit * len(states))()
        for k, st in enumerate(states):
            arrs = [np.ascontiguousarray(getattr(st, f), dtype=np.float64)
                    for f in ("r", "v", "q", "p", "m", "I")]
            self._keep.append(arrs)
            ri = inits[k]
            ri.r, ri.v, ri.q, ri.p, ri.mass, ri.inertia = [_p(a) for a in arrs]
            ri.s, ri.Ps, ri.Q, ri.W, ri.T, ri.P = st.s, st.Ps, st.Q, st.W, st.T, st.P
            for x in range(3):
                ri.Pv[x] = st.Pv[x]
                ri.L[x] = st.L[x]
        self.nrep = len(states)
        self.nmol = np.array([st.nmol for st in states])
        self.h = C.c_void_p()
        prec = 1 if precision == "fp64" else 0
        _check(L.remd_create((SystemDesc * n_e)(*descs), n_e, _p(self.reps_per_ens, _ip), inits,
                             prec, device, C.byref(self.h)))
        self._keep = None
        self.T = np.array([st.T for st in states])
        self.P = np.array([st.P for st in states])

    def close(self):
        if self.h:
            lib().remd_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- REMDGPU surface
    def ExecuteSteps(self, T, P):
        T = np.ascontiguousarray(T, dtype=np.float64)
        P = np.ascontiguousarray(P, dtype=np.float64)
        _check(lib().remd_execute_steps(self.h, _p(T), _p(P)))
        self.T, self.P = T.copy(), P.copy()

    def GetAverages(self, rep):
        out = np.zeros(NUM_AVG)
        _check(lib().remd_get_averages(self.h, rep, _p(out)))
        return out

    def all_averages(self):
        out = np.zeros((self.nrep, NUM_AVG))
        _check(lib().remd_get_all_averages(self.h, _p(out)))
        return out

    def ConvertVariablesToHost(self, rep):
        n = int(self.nmol[rep])
        arrs = dict(r=np.zeros((n, 3)), v=np.zeros((n, 3)), q=np.zeros((n, 4)),
                    p=np.zeros((n, 4)), f=np.zeros((n, 3)), n=np.zeros((n, 4)))
        sv = StateView()
        for k, a in arrs.items():
            setattr(sv, k, _p(a))
        _check(lib().remd_get_state(self.h, rep, C.byref(sv)))
        out = dict(arrs)
        out.update(s=sv.s, Ps=sv.Ps, Q=sv.Q, Pv=np.array(sv.Pv[:]), W=sv.W, L=np.array(sv.L[:]),
                   T=sv.T, P=sv.P, H0=sv.H0, pot=sv.pot, lj=sv.lj, clmb=sv.clmb, wall=sv.wall,
                   vir=np.array(sv.vir[:]))
        return out

    def state(self, rep) -> ReplicaState:
        g = self.ConvertVariablesToHost(rep)
        n = int(self.nmol[rep])
        return ReplicaState(g["r"], g["v"], g["q"], g["p"], np.zeros(n), np.zeros((n, 3)),
                            g["s"], g["Ps"], g["Q"], g["Pv"], g["W"], g["L"], g["T"], g["P"])

    # ---- engine extras
    def execute_nsteps(self, n):
        _check(lib().remd_execute_nsteps(self.h, n))

    def rescale_velocities(self):
        """The reference's init_scaling (VelocityScaling + AngVelocityScaling)."""
        _check(lib().remd_rescale_velocities(self.h))

    def equilibrate(self, rounds=10, steps=20):
        """Relax a lattice start: `rounds` x (`steps` MD steps, then init_scaling)."""
        for _ in range(rounds):
            self.execute_nsteps(steps)
            self.rescale_velocities()

    def replica_pair_count(self, rep):
        return int(lib().remd_replica_pair_count(self.h, rep))

    def compute_forces(self):
        _check(lib().remd_compute_forces(self.h))

    def pair_count(self):
        return int(lib().remd_last_pair_count(self.h))

    def launches_per_interval(self):
        return int(lib().remd_launches_per_interval(self.h))

    def set_tuning(self, tile, skin):
        _check(lib().remd_set_tuning(self.h, tile, skin))

    def autotune(self, nsteps=20):
        """Pick the fastest (tile, skin) for this batch (remd_autotune); the
        trajectory does not depend on the choice.  Returns (tile, skin, ms per step)."""
        t, k, ms = C.c_int(), C.c_double(), C.c_double()
        _check(lib().remd_autotune(self.h, nsteps, C.byref(t), C.byref(k), C.byref(ms)))
        return t.value, k.value, ms.value

    def execute_async(self, T=None, P=None):
        if T is None:
            _check(lib().remd_execute_steps_async(self.h, None, None))
        else:
            T = np.ascontiguousarray(T, dtype=np.float64)
            P = np.ascontiguousarray(P, dtype=np.float64)
            _check(lib().remd_execute_steps_async(self.h, _p(T), _p(P)))

    def synchronize(self):
        _check(lib().remd_synchronize(self.h))

    def replica_status(self, rep):
        s = C.c_int()
        _check(lib().remd_replica_status(self.h, rep, C.byref(s)))
        return s.value

    def exchange_device(self, grids, step, u=None, seed=0):
        g = np.ascontiguousarray(grids, dtype=np.int32).reshape(-1)
        up = _p(np.ascontiguousarray(u, dtype=np.float64)) if u is not None else None
        _check(lib().remd_exchange_device(self.h, _p(g, _ip), step, up, seed))

    def enable_device_exchange(self, grids, seed=0, first_step=0):
        """Run the Metropolis exchange on the device after every interval."""
        if grids is None:
            _check(lib().remd_enable_device_exchange(self.h, None, 0, 0))
            return
        g = np.ascontiguousarray(grids, dtype=np.int32).reshape(-1)
        _check(lib().remd_enable_device_exchange(self.h, _p(g, _ip), seed, first_step))

    def execute_device(self):
        _check(lib().remd_execute_steps_device(self.h))

    def conditions(self):
        idx = np.zeros(self.nrep, dtype=np.int32)
        T, P = np.zeros(self.nrep), np.zeros(self.nrep)
        _check(lib().remd_get_conditions(self.h, _p(idx, _ip), _p(T), _p(P)))
        return idx, T, P

    # ---- (volume, potential) histograms (REMDInfo's Histogram)
    def histogram_enable(self, ens, energy_min, energy_max, volume_min, volume_max):
        _check(lib().remd_histogram_enable(self.h, ens, C.c_double(energy_min), C.c_double(energy_max),
                                           C.c_double(volume_min), C.c_double(volume_max)))

    def histogram_increment(self, index=None):
        """REMD::IncrementHistogram; index: slot -> replica, ensemble-local,
        ensembles concatenated (None: the engine's own index)."""
        if index is None:
            _check(lib().remd_histogram_increment(self.h, None))
        else:
            idx = np.ascontiguousarray(index, dtype=np.int32)
            _check(lib().remd_histogram_increment(self.h, _p(idx, _ip)))

    def histogram(self, ens, slot):
        """(bounds {vmin, vmax, pmin, pmax, samples}, counts (500, 500), per-bin sums (500, 500, 19))."""
        b = np.zeros(5, dtype=np.int32)
        hist = np.zeros((500, 500), dtype=np.int32)
        ave = np.zeros((500, 500, 19))
        _check(lib().remd_histogram_get(self.h, ens, slot, _p(b, _ip), _p(hist, _ip), _p(ave)))
        return b, hist, ave

    def histogram_write(self, ens, directory):
        _check(lib().remd_histogram_write(self.h, ens, directory.encode()))

    def histogram_read(self, ens, directory):
        _check(lib().remd_histogram_read(self.h, ens, directory.encode()))

    def write_chk(self, rep, path):
        _check(lib().remd_write_chk(self.h, rep, path.encode()))

    def OutputCDV(self, prefix, step):
        """REMDGPU::OutputCDV: a <prefix>R%04ds%07d.cdv snapshot of every replica
        (remd_output_cdv)."""
        _check(lib().remd_output_cdv(self.h, prefix.encode(), C.c_uint(step)))

    def write_gro(self, rep, path, moltype):
        """The reference's .gro output of replica rep (remd_write_gro); names from
        the molecule type."""
        names = (C.c_char_p * moltype.nsite)(*[a.encode() for a in moltype.names])
        _check(lib().remd_write_gro(self.h, rep, path.encode(), moltype.name.encode(), names))


def force_snapshot_noalloc(spec, d_r, d_q, L, d_wall, d_f, d_n, d_out, stream=None):
    """remd_force_snapshot_noalloc on caller-owned device buffers (addresses as
    ints): for callers that cannot let the library allocate device memory.
    Asynchronous on `stream` (a cudaStream_t as int, None = default stream)."""
    d = system_desc(spec)
    Lh = np.ascontiguousarray(L, dtype=np.float64)
    _check(lib().remd_force_snapshot_noalloc(C.byref(d), d_r, d_q, _p(Lh), d_wall or None, d_f, d_n,
                                             d_out, stream))


def wall_table(confined, nfwall, wall_length, sgm, eps, rho):
    out = np.zeros(2 * nfwall)
    _check(lib().remd_wall_table(confined, nfwall, wall_length, sgm, eps, rho, _p(out)))
    return out.reshape(nfwall, 2)


def read_chk(path, nmol):
    r, v, I = np.zeros((nmol, 3)), np.zeros((nmol, 3)), np.zeros((nmol, 3))
    q, p, m, sc = np.zeros((nmol, 4)), np.zeros((nmol, 4)), np.zeros(nmol), np.zeros(10)
    _check(lib().remd_read_chk(path.encode(), nmol, _p(r), _p(v), _p(q), _p(p), _p(m), _p(I),
                               _p(sc)))
    return ReplicaState(r, v, q, p, m, I, sc[0], sc[1], sc[2], sc[3:6].copy(), sc[6],
                        sc[7:10].copy())


def write_chk_arrays(path, nsite, st: ReplicaState, prop):
    """IOManager::WriteCheckPoint from host arrays (remd_write_chk_arrays): the
    state in the remd_read_chk convention and the 26 Property-line numbers."""
    f = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    n = len(st.r)
    sc = f([st.s, st.Ps, st.Q, *st.Pv, st.W, *st.L])
    _check(lib().remd_write_chk_arrays(path.encode(), n, nsite, _p(f(st.r)), _p(f(st.v)), _p(f(st.q)),
                                       _p(f(st.p)), float(st.m[0]), _p(f(st.I[0])), _p(sc),
                                       _p(f(prop))))


def exchange_host(ntemp, npress, pconstant, step, index, T, P, pot, vol, u):
    """REMD::ReplicaExchange on the host (in place); returns accept flags."""
    acc = np.zeros(max(ntemp * npress // 2, 1), dtype=np.int32)
    npairs = C.c_int()
    _check(lib().remd_exchange_host(ntemp, npress, pconstant, step, _p(index, _ip), _p(T), _p(P),
                                    _p(np.ascontiguousarray(pot, dtype=float)),
                                    _p(np.ascontiguousarray(vol, dtype=float)),
                                    _p(np.ascontiguousarray(u, dtype=float)), _p(acc, _ip),
                                    C.byref(npairs)))
    return acc[:npairs.value].copy()
