/*
 * remd_b200.h -- C-ABI of the B200 REMD engine (libremd_b200.so).
 *
 * The engine replaces the reference's GPU engine, class REMDGPU
 * (src/remdgpu.h:92-238), and the CPU surface the REMD driver uses on the hot
 * path (Molecules::ExecuteSteps / GetAverage / ChangeTemperature ...,
 * src/molecules.h:305-402).  Every call returns a remd_status; none exits the
 * process (the reference calls exit(EXIT_FAILURE), src/remdgpu.cu:208-212).
 *
 * Units are the reference's reduced units (src/unit.h:1-19): length A, energy
 * kJ/mol, mass 15.9994 g/mol, time sqrt(m A^2 / E); temperatures and pressures
 * passed in and out are reduced (T/unit_temp, P/unit_press), exactly what
 * REMDInfo::temperature / pressure hold (src/remdinfo.cxx:167-170).
 *
 * Replica state uses Molecules' internal convention after ReadCheckPoint
 * (src/io_manager.cxx:580-585): r is the box fraction in [0,1), v is the
 * velocity multiplied by L*s, p the conjugate quaternion momentum multiplied
 * by s.
 *
 * Threading: one handle is used by one host thread at a time.  Device work is
 * issued on the handle's own CUDA stream; calls that return host data
 * synchronise that stream.
 */
#ifndef REMD_B200_H
#define REMD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  REMD_OK = 0,
  REMD_ERR_INVALID = 1,        /* bad argument or unsupported combination            */
  REMD_ERR_OOM = 2,            /* device allocation or HBM budget exceeded           */
  REMD_ERR_TIMEOUT = 3,        /* a bounded wait ran out                             */
  REMD_ERR_NONFINITE = 4,      /* a replica produced NaN/Inf (see remd_replica_status)*/
  REMD_ERR_CANCELLED = 5,      /* job cancelled                                      */
  REMD_ERR_CUDA = 6,           /* CUDA runtime error (message in remd_last_error)    */
  REMD_ERR_IO = 7,             /* file could not be read or written                  */
  REMD_ERR_NEIGHBOR_OVERFLOW = 8, /* a neighbour list exceeded its capacity          */
  REMD_ERR_NO_DEVICE = 9,      /* no CUDA device                                     */
  REMD_ERR_RANGE = 10          /* a histogram sample fell outside its range          */
} remd_status;

#define REMD_NUM_AVERAGES 19   /* Average::NUM_ELEM, src/remdinfo.h:29-41 */
#define REMD_MAX_SITES 5

/* Average field order (src/remdinfo.h:29-41): */
enum {
  REMD_AVG_LJ = 0, REMD_AVG_CLMB, REMD_AVG_WALL, REMD_AVG_VOL, REMD_AVG_TRA, REMD_AVG_ROT,
  REMD_AVG_T, REMD_AVG_P, REMD_AVG_PX, REMD_AVG_PY, REMD_AVG_PZ, REMD_AVG_TOT, REMD_AVG_DRF,
  REMD_AVG_TSTS, REMD_AVG_TSTV, REMD_AVG_BSTX, REMD_AVG_BSTY, REMD_AVG_BSTZ, REMD_AVG_DUMMY
};

/* Force arithmetic of a handle. */
typedef enum {
  REMD_PREC_FP32 = 0,   /* FP32 pair math, FP64 per-molecule/replica accumulation */
  REMD_PREC_FP64 = 1    /* all-FP64 (the plain form)                            */
} remd_precision;

/* One REMD system (an "ensemble"): the Parameter fields on the path
 * (src/parameter.h:9-300) plus its molecule type as read from moltype.txt
 * (src/molecules.cxx:69-131; A, g/mol, A, kJ/mol, e).  Site 0 must be the only
 * Lennard-Jones site (water oxygen); the charged sites must be contiguous and
 * end at the last site. */
typedef struct {
  int nmol;
  int nsite;
  double site_r[REMD_MAX_SITES][3];
  double site_mass[REMD_MAX_SITES];
  double site_sigma[REMD_MAX_SITES];
  double site_eps[REMD_MAX_SITES];
  double site_charge[REMD_MAX_SITES];
  int tconstant;            /* 0 NVE-like, 1 Nose-Poincare, 2 velocity scaling  */
                            /* before every step (bulk pconstant 0; tube         */
                            /* pconstant 0 or 2: Molecules::ExecuteSteps,        */
                            /* src/integrator.cxx:713-787)                       */
  int pconstant;            /* 0 none, 1 3-D, 2 z (tube), 3 xy (slit)            */
  int confined;             /* 0 bulk, 1 nanotube, 2 nano-slit                   */
  double dt_fs;
  double rcut, rswitch;     /* A */
  int nfwall;               /* wall table entries, 3 .. 16777216 (confined only)  */
  double wall_length;       /* A: tube radius or slit width                       */
  double sgm_wall, eps_wall, rho_wall;
  int interval;             /* MD steps per ExecuteSteps call                    */
} remd_system_desc;

/* Initial state of one replica (borrowed for the duration of the call). */
typedef struct {
  const double *r;          /* nmol*3 box fraction                               */
  const double *v;          /* nmol*3 velocity * L * s                           */
  const double *q;          /* nmol*4 unit quaternion                            */
  const double *p;          /* nmol*4 conjugate momentum * s                     */
  const double *mass;       /* nmol   reduced mass (the .chk "m" column)         */
  const double *inertia;    /* nmol*3 principal moments (the .chk "I" columns)   */
  double s, Ps, Q;          /* Thermostat, src/variables.h:260-271               */
  double Pv[3], W;          /* Barostat, src/variables.h:273-280                 */
  double L[3];              /* box lengths, A                                    */
  double T, P;              /* reduced condition                                 */
} remd_replica_init;

/* Mutable view filled by remd_get_state (caller-owned arrays, any may be NULL). */
typedef struct {
  double *r, *v, *q, *p;    /* as remd_replica_init                              */
  double *f;                /* nmol*3 molecular force of the last force call      */
  double *n;                /* nmol*4 body torque 4-vector (src/molecules.cxx:409-418) */
  double s, Ps, Q, Pv[3], W, L[3], T, P, H0;
  double pot, lj, clmb, wall, vir[3];
} remd_state_view;

typedef struct remd_engine_s *remd_handle;

/* ---- engine lifetime ------------------------------------------------------ */

/* Replaces REMDGPU::REMDGPU(Molecules**, nreplica) (src/remdgpu.cu:178-503).
 * nens systems; reps_per_ens[e] replicas of system e, their states in order in
 * reps.  Computes the initial forces and H0 (the reference's dt=0 pass,
 * src/remdgpu.cu:461-478).  All systems must share `interval`. */
remd_status remd_create(const remd_system_desc *systems, int nens, const int *reps_per_ens,
                        const remd_replica_init *reps, remd_precision prec, int device,
                        remd_handle *out);

/* Replaces REMDGPU::~REMDGPU. */
remd_status remd_destroy(remd_handle h);

/* Replaces REMDGPU::ExecuteSteps(double* T, double* P) (src/remdgpu.cu:656-681):
 * advance every replica by `interval` steps under the given reduced conditions
 * (length = total replicas).  A replica whose T or P differs from its previous
 * condition first gets the reference's exchange tail (ChangeTemperature,
 * KillMomentum, SetPressure, CalcProperties, UpdateHamiltonian,
 * src/remd.cxx:526-536). */
remd_status remd_execute_steps(remd_handle h, const double *T, const double *P);

/* Same, with the conditions already on the device and without the trailing
 * copy of the averages (used by remd_run_remd and the benchmark). */
remd_status remd_execute_steps_async(remd_handle h, const double *T, const double *P);
remd_status remd_synchronize(remd_handle h);

/* Advance every replica by nsteps MD steps (kernels launched one by one; the
 * interval start/end bookkeeping as in remd_execute_steps, conditions as left
 * by the last call).  Molecules::ExecuteSteps with interval = nsteps
 * (src/integrator.cxx:708-803). */
remd_status remd_execute_nsteps(remd_handle h, int nsteps);

/* The reference's init_scaling for every replica: Molecules::VelocityScaling
 * and AngVelocityScaling (src/molecules.cxx:262-307) -- kinetic energies set to
 * 1.5 N T, momentum removed, s=1, Ps=0, Pv=0 -- then H0 recomputed as in
 * InitializeProperty (src/molecules.h:260-270).  v and p are first divided by
 * s (a no-op at start-up, where the reference calls it with s = 1). */
remd_status remd_rescale_velocities(remd_handle h);

/* Replaces REMDGPU::GetAverages(rep) (src/remdgpu.h:208-233): the 19 fields of
 * Average for replica `rep` after the last ExecuteSteps (T and P reduced). */
remd_status remd_get_averages(remd_handle h, int rep, double out[REMD_NUM_AVERAGES]);
/* All replicas at once: out is nrep*19. */
remd_status remd_get_all_averages(remd_handle h, double *out);

/* Replaces REMDGPU::ConvertVariablesToHost (src/remdgpu.cu:806-854). */
remd_status remd_get_state(remd_handle h, int rep, remd_state_view *out);

/* Recompute forces (no integration) and return them through remd_get_state:
 * the snapshot used by the parity tests (Molecules::CalcForcePot). */
remd_status remd_compute_forces(remd_handle h);

/* Totals and per-replica information. */
int remd_num_replicas(remd_handle h);
int remd_replica_nmol(remd_handle h, int rep);
/* Unordered molecule pairs within rcut evaluated by the last force call, summed
 * over replicas (integer reduction; the roofline's pair count). */
long long remd_last_pair_count(remd_handle h);
/* Number of the engine's kernels launched per ExecuteSteps call. */
int remd_launches_per_interval(remd_handle h);

/* Unordered pairs within rcut of one replica in the last force call. */
long long remd_replica_pair_count(remd_handle h, int rep);

/* The handle's CUDA stream (a cudaStream_t), for timing with CUDA events. */
void *remd_stream(remd_handle h);

/* Timing pass: runs nsteps MD steps launching the kernels one by one (no
 * graph) with CUDA events around each launch, and returns the mean device
 * time in ms of {integrate, force} launches in ms_out[0..1].  The state
 * advances like remd_execute_steps minus the interval start/end kernels'
 * bookkeeping (use on a scratch handle). */
remd_status remd_profile_steps(remd_handle h, int nsteps, double *ms_out);

/* remd_profile_steps with the force step split per launch: ms_out[0..3] the
 * mean time per MD step of the integrate kernel, the replica head, the list
 * kernel and the pair kernel (FP64 form: [2] = 0, [3] its one force kernel);
 * ms_out[4] the mean number of replicas whose neighbour lists were rebuilt per
 * step.  One launch chain, CUDA events between the launches. */
remd_status remd_profile_split(remd_handle h, int nsteps, double *ms_out);

/* FP32 FMA throughput of this GPU (TFLOP/s, FMA = 2 flops) from a register-
 * resident FMA-chain kernel over every SM; the denominator of the force
 * kernel's roofline. */
remd_status remd_measure_fp32_peak(int device, double *tflops);

/* Integer-add throughput of this GPU in G adds/s, rates[0..3]: 64-bit into
 * shared memory, 32-bit into shared memory, 64-bit into the shared memory of
 * a peer block of a four-block cluster, 64-bit into global memory (L2).  Each
 * of 4 blocks x 512 threads per SM adds to pseudo-random words of a 41 KB
 * array (7 values x 736 molecules).  The rates at which a pair kernel that
 * computes each pair once could add the partner's share in fixed point. */
remd_status remd_measure_atomics(int device, double *rates);

/* Per-replica health word of the last interval: 0 ok, else a remd_status. */
remd_status remd_replica_status(remd_handle h, int rep, int *status);

/* Tuning: molecules of one force tile (multiple of 32: 32..64 for FP32 handles,
 * 32..128 for FP64; defaults 32 / 128) and the neighbour
 * skin (A).  Takes effect on the next call. */
remd_status remd_set_tuning(remd_handle h, int tile, double skin);

/* Autotuner (no counterpart in the reference): times every (tile, skin) of
 * {32, 64, 96, 128} x {0.6, 0.8, 1.0, 1.4} A that the handle's precision
 * allows (remd_set_tuning) over `nsteps` MD steps of this
 * batch (integrate + force per step, CUDA events), restores the state after
 * each trial and keeps the fastest.  The trajectory does not depend on the
 * choice: forces are a function of positions only and every partial sum is
 * per 32 molecules.  Outputs (any may be NULL): the chosen tile, skin and its
 * ms per MD step.  Synchronous; call it before stream capture. */
remd_status remd_autotune(remd_handle h, int nsteps, int *tile, double *skin, double *ms_per_step);

/* ---- exchange (src/remd.cxx:467-538, src/remdinfo.cxx:54-125) ------------- */

/* REMD::ReplicaExchange for one ensemble on the host: index (condition slot ->
 * replica), temperature/pressure (per replica) are updated in place; u[i] is
 * the uniform compared with exp(-delta) for pair i of list step%4.  Writes the
 * accept flags (length ntemp*npress/2) and returns the pair count in *npairs. */
remd_status remd_exchange_host(int ntemp, int npress, int pconstant, long step, int *index,
                               double *temperature, double *pressure, const double *pot,
                               const double *vol, const double *u, int *accepted,
                               int *npairs);

/* The same decision for every ensemble of a handle, on the device, fed by the
 * potential energies and volumes of the last interval.  u holds, per ensemble,
 * ntemp*npress/2 uniforms (concatenated); pass NULL to draw them from a
 * counter-based Philox stream seeded with `seed`.  grids gives ntemp,npress per
 * ensemble (2*nens ints).  Conditions take effect on the next
 * remd_execute_steps_device call. */
remd_status remd_exchange_device(remd_handle h, const int *grids, long step, const double *u,
                                 unsigned long long seed);
/* Advance one interval with the conditions left on the device by
 * remd_exchange_device (no host round trip). */
remd_status remd_execute_steps_device(remd_handle h);
/* Append the Metropolis exchange of every ensemble to each interval run by
 * remd_execute_steps_async/_device (one REMD interval = interval MD steps +
 * the exchange, REMD::ExecuteREMD, src/remd.cxx:297-441), with a per-ensemble
 * step counter starting at first_step and Philox uniforms from seed.  grids =
 * NULL turns it off.  Conditions chosen by the exchange are applied at the
 * start of the next interval. */
remd_status remd_enable_device_exchange(remd_handle h, const int *grids, unsigned long long seed,
                                        long long first_step);
/* Read back the device-side condition arrays (index per ensemble slot, T, P per replica). */
remd_status remd_get_conditions(remd_handle h, int *index, double *T, double *P);

/* ---- host-side formats ----------------------------------------------------- */

/* ForceCalculator::CalcWallForce (src/force_calculator.cxx:117-200): the
 * nfwall x {f, U} wall table the engine builds at create. */
remd_status remd_wall_table(int confined, int nfwall, double wall_length, double sgm_wall,
                            double eps_wall, double rho_wall, double *out);

/* IOManager::ReadCheckPoint (src/io_manager.cxx:528-591): reads a .chk into
 * caller arrays sized for nmol (r, v, q, p, mass, inertia converted like the
 * reference; scal = s Ps Q Pv0 Pv1 Pv2 W L0 L1 L2). */
remd_status remd_read_chk(const char *path, int nmol, double *r, double *v, double *q, double *p,
                          double *mass, double *inertia, double *scal);
/* IOManager::WriteCheckPoint (src/io_manager.cxx:593-634) of replica rep, with
 * the reference's text layout byte for byte.  The last line is the replica's
 * Property (src/variables.h:51-74) as the engine holds it after the last call:
 * time = MD steps run by the handle x dt, the energies and pressures of the
 * last interval's averages (or of the initial force call), the momentum and the
 * virial of the current state; the running averages Tave and Pave are those of
 * the last property evaluation alone (the reference's nave = 1). */
remd_status remd_write_chk(remd_handle h, int rep, const char *path);
/* IOManager::WriteCheckPoint (src/io_manager.cxx:593-634) from host arrays in the
 * remd_read_chk convention (r box fraction, v * L * s, p * s, nmol rows each;
 * mass and inertia[3], the principal moments, shared by every molecule;
 * scal = s Ps Q Pv0 Pv1 Pv2 W L0 L1 L2).
 * prop holds the 26 numbers of the Property line in its operator<< order
 * (src/variables.h:51-74): time pot tra rot kin tsm tsp tst bst tot ham, tmo[3],
 * Tave/nave, prs[4], vir[3], Pave[4]/nave. */
remd_status remd_write_chk_arrays(const char *path, int nmol, int nsite, const double *r,
                                  const double *v, const double *q, const double *p, double mass,
                                  const double *inertia, const double *scal, const double *prop);
/* The .gro output of replica rep as IOManager::UpdateOutputs writes it
 * (src/io_manager.cxx:636-651 -> ConvertMoleculesToAtoms 797-814 ->
 * write_gro_file, src/gro.cxx:118-135): comment "test", site coordinates
 * r L + R(q) b in nm, velocities 0, box in nm.  The molecule and site names
 * (moltype.txt; the engine does not keep them) are padded to 5 characters like
 * MakeMolTypeList does (src/molecules.cxx:86, 95). */
remd_status remd_write_gro(remd_handle h, int rep, const char *path, const char *mol_name,
                           const char *const *atom_names);
/* REMDGPU::OutputCDV (src/remdgpu.cu:700-804): a CDView snapshot of every
 * replica to <prefix>R%04d s%07d .cdv (rep, step): box (tube: +-wall_length in
 * x, y; slit: +-wall_length/2 in z), colours, "T=.. K, P=.. MPa", then one line
 * "mol site x y z" per site in A from the box centre, in the reference's single
 * precision. */
remd_status remd_output_cdv(remd_handle h, const char *prefix, unsigned int step);

/* ---- (volume, potential) histograms on the device ------------------------- */
/* REMDInfo's per-condition histograms (src/remdinfo.h:93-139, 299-331; 500 x 500
 * bins, linear sampling), kept on the device for ensemble ens: one per condition
 * slot, with the 19 Average fields summed per bin.  energy in kJ/mol and volume
 * in A^3, both per molecule (the .inp energy_min/max, volume_min/max).  Enabling
 * again clears it.  About 39 MB of device memory per condition slot. */
remd_status remd_histogram_enable(remd_handle h, int ens, double energy_min, double energy_max,
                                  double volume_min, double volume_max);
/* REMD::IncrementHistogram (src/remd.cxx:803-813) after an interval: the slot c
 * histogram of each ensemble gets the sample of the replica index[c] holds
 * (ensemble-local indices, ensembles concatenated like the replicas).  index
 * NULL: the engine's own index (the device exchange's).  With the device
 * exchange enabled the interval graph already does this before exchanging; do
 * not call it then.  A sample out of range returns REMD_ERR_RANGE (the
 * reference exits). */
remd_status remd_histogram_increment(remd_handle h, const int *index);
/* One slot's histogram: bounds = {vmin, vmax, pmin, pmax, samples}, hist the
 * 500 x 500 counts (volume-major), ave the 500 x 500 x 19 per-bin sums; any may
 * be NULL. */
remd_status remd_histogram_get(remd_handle h, int ens, int slot, int *bounds, int *hist, double *ave);
/* REMDInfo::OutputHistogram (src/remdinfo.cxx:723-758): dir/histo_P%lf_T%lf.dat
 * per slot, with the slot's reduced condition. */
remd_status remd_histogram_write(remd_handle h, int ens, const char *dir);
/* REMDInfo::ReadHistogramFromBackUp (src/remdinfo.cxx:681-721) from those files. */
remd_status remd_histogram_read(remd_handle h, int ens, const char *dir);

/* Force snapshot of one replica that allocates nothing.  No counterpart in the
 * reference: it exists for callers that cannot allocate device memory -- a host
 * program whose own allocator already owns the GPU (an ML framework's caching
 * allocator, a plugin host), or a loop that must not stall on cudaMalloc /
 * cudaFree, which can synchronise the device.  The caller passes device
 * buffers: d_r (nmol*3 box fractions), d_q (nmol*4 quaternions), d_wall (the
 * nfwall x {f,U} table from remd_wall_table, 16-byte aligned; NULL for bulk),
 * and receives d_f (nmol*3 forces), d_n (nmol*4 body torques) and d_out[8] =
 * {LJ, Coulomb, wall, virial x3, unordered pairs within rcut, error word (0 ok,
 * 1 neighbour overflow)}; L is the host box.  Same FP32 arithmetic as a
 * REMD_PREC_FP32 handle's remd_compute_forces.  All working memory is one
 * fixed device array of the library (about 8.8 MB, held by every GPU that
 * loads it until exit): at most 2048 molecules and 1024 neighbours per molecule
 * (rcut <= ~12.4 A); larger inputs are rejected with REMD_ERR_INVALID, and so
 * are a d_wall that is not 16-byte aligned and other buffers that are not
 * 8-byte aligned.  The first call on a device looks up that array's device
 * address (set-up) and keeps it for the process, so make it before any stream
 * capture, and make no call after a cudaDeviceReset of that device (the reset
 * reloads the library's module, and the kept address may no longer be the
 * array's).  The constants of a call travel as kernel parameters, so no host
 * buffer has to outlive the call.  Calls share the array and keep the previous
 * call's contents, so calls that overlap on the GPU (other streams, other
 * threads) race; serialise them.  Asynchronous on `stream` (a cudaStream_t,
 * NULL = default stream). */
remd_status remd_force_snapshot_noalloc(const remd_system_desc *sys, const double *d_r,
                                        const double *d_q, const double L[3], const double *d_wall,
                                        double *d_f, double *d_n, double *d_out, void *stream);

/* Text of the last error on this thread. */
const char *remd_last_error(void);
/* Library version string. */
const char *remd_version(void);

/* ---- serving: continuous batching of REMD jobs ----------------------------- */

typedef struct remd_server_s *remd_server;
typedef long long remd_job_id;

typedef struct {
  remd_system_desc system;
  int ntemp, npress;
  const remd_replica_init *reps;   /* ntemp*npress states, copied at submit */
  int ninterval;                   /* intervals to run                       */
  unsigned long long seed;         /* exchange stream                        */
} remd_job_desc;

typedef struct {
  int state;                 /* 0 queued, 1 running, 2 done, 3 failed, 4 cancelled */
  int intervals_done;
  double submit_s, start_s, end_s;   /* server clock, seconds */
  remd_status status;
} remd_job_info;

typedef struct {
  long long jobs_done, intervals_done, mol_steps;
  double p50_interval_ms, p99_interval_ms;   /* per round: admission, batch change, interval */
  double p50_job_s, p99_job_s;               /* submit -> done                               */
  double busy_s;
  long long bytes_in_use, budget_bytes;
  long long batch_changes;                   /* rounds that built a new batch handle         */
  double max_batch_change_ms;                /* slowest of those builds                      */
  double max_graph_ms;                       /* slowest interval-graph capture + update      */
} remd_server_stats;

remd_status remd_server_open(size_t hbm_budget_bytes, int device, remd_precision prec,
                             remd_server *out);
remd_status remd_server_close(remd_server s);
remd_status remd_job_submit(remd_server s, const remd_job_desc *job, remd_job_id *id);
remd_status remd_job_poll(remd_server s, remd_job_id id, remd_job_info *info);
remd_status remd_job_cancel(remd_server s, remd_job_id id);
/* Final averages (ntemp*npress*19) and the condition index of a finished job. */
remd_status remd_job_result(remd_server s, remd_job_id id, double *averages, int *index);
/* Run one scheduling round: admit queued jobs while the budget allows, then
 * advance every admitted job by one interval as one batch.  Returns the number
 * of jobs still queued or running in *pending. */
remd_status remd_server_step(remd_server s, int *pending);
remd_status remd_server_stats_get(remd_server s, remd_server_stats *out);
/* The device footprint the server budgets for a job (the engine's layout formula). */
remd_status remd_job_bytes(const remd_job_desc *job, size_t *bytes);

#ifdef __cplusplus
}
#endif
#endif /* REMD_B200_H */
