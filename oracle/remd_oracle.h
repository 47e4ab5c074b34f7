/*
 * remd_oracle.h -- CPU restatement, in plain C99 and FP64, of the subarutaro/remd
 * hot path: switched-cutoff LJ + Coulomb rigid-water forces, the tabulated
 * nanotube / slit wall, the Nose-Poincare / Andersen quaternion integrator,
 * the observables and the Metropolis T/P exchange.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the CUDA
 * engine.  Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * reference arm may load it; the engine never calls it.
 *
 * Pinning: for bulk (confined=0) and nanotube (confined=1) systems every
 * function here is checked against the reference's own CPU sources, compiled
 * unmodified into oracle/_ref (see oracle/Makefile and oracle/ref_driver.cxx),
 * and against the reference's golden line test/correct:4.  The slit
 * (confined=2) wall and 2-D barostat cannot be pinned that way: the reference
 * CPU slit branch is broken (src/force_calculator.cxx:1556-1561, and the tuned
 * branch asserts at :1525) and its GPU slit kernel does not compile on CUDA 12.
 * For confined=2 this file restates the reference GPU kernel's semantics
 * (src/remdgpu.cu:1708-1720 wall, 2083-2120 D4, 2529-2555 D5); that part is
 * "parity unpinned".
 *
 * Units are the reference's reduced units (src/unit.h:1-19): length 1 A,
 * energy 1 kJ/mol, mass 15.9994 g/mol, time sqrt(m A^2 / E).
 */
#ifndef REMD_ORACLE_H
#define REMD_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_NSITE_MAX 5
#define ORC_NUM_AVG 19

/* unit constants restated from src/unit.h:1-19 */
double orc_unit_time(void);
double orc_unit_temp(void);
double orc_unit_press(void);
double orc_unit_coulomb(void);
double orc_unit_mass(void);

/* One rigid molecule type after MakeMolTypeList's normalisation
 * (src/molecules.cxx:69-131) and MakeParamList's mixing (src/force_calculator.cxx:203-244). */
typedef struct {
  int nsite;
  double body[ORC_NSITE_MAX][3];     /* site offsets in the body frame */
  double mass[ORC_NSITE_MAX];
  double sgm2[ORC_NSITE_MAX][ORC_NSITE_MAX]; /* ((s_i+s_j)/2)^2 */
  double eps[ORC_NSITE_MAX][ORC_NSITE_MAX];  /* sqrt(e_i e_j) */
  double q[ORC_NSITE_MAX];
  double inertia[3];                 /* MolType::CalcIner, src/variables.h:316-334 */
} orc_moltype;

/* Build a molecule type from moltype.txt values (A, g/mol, A, kJ/mol, e). */
void orc_moltype_from_input(orc_moltype *mt, int nsite, const double *r /*nsite*3*/,
                            const double *mass, const double *sigma,
                            const double *eps, const double *charge);

/* The per-system constants one Molecules object holds. */
typedef struct {
  int nmol;
  int tconstant, pconstant, confined;
  double dt, dthalf;          /* reduced time */
  double rcut, rswitch;       /* A */
  int nfwall;
  double wall_length_param;   /* A, as read from .inp */
  double wall_length;         /* reduced, ForceCalculator::wall_length */
  double *fwall;              /* nfwall x {f, U}; caller-owned */
  orc_moltype mt;
} orc_system;

/* Fill the time/wall fields of sys from .inp values (dt in fs, wall in A). */
void orc_system_init(orc_system *sys, int nmol, int tconstant, int pconstant,
                     int confined, double dt_fs, double rcut, double rswitch,
                     int nfwall, double wall_length_A);

/* Replica state: the fields of Molecule/Thermostat/Barostat/Property the path uses
 * (src/variables.h:216-284).  r is the box fraction in [0,1), v is scaled by L*s,
 * p by s, exactly as Molecules stores them after ReadCheckPoint. */
typedef struct {
  double *r, *v, *q, *p, *f, *n;   /* nmol*3, *3, *4, *4, *3, *4 */
  double *m;                       /* nmol */
  double *I;                       /* nmol*3 */
  double *ar, *af;                 /* scratch: nmol*nsite*3 each */
  double s, Ps, Q;
  double Pv[3], W;
  double L[3];
  double T, P;                     /* reduced */
  double gkT, H0;
  double pot, lj, clmb, wall, vir[3];
  double tra3[3], tra, rot, kin, Tk, prs[4], tsm, tsp, tst, bst, tot, ham;
  long long npairs;                /* unordered COM pairs within rcut in the last force call */
} orc_replica;

/* ForceCalculator::CalcWallForce, src/force_calculator.cxx:117-200.
 * fwall is nfwall x {f, U}.  sgm_A, eps_kJ, wall_A as read from .inp. */
void orc_wall_table(int confined, int nfwall, double wall_A, double sgm_A,
                    double eps_kJ, double rho, double *fwall);

/* Molecules::CalcForcePot for the generic switched build (no *_SITE macro):
 * ConvertToAtoms + ForceCalculator::Switching + Confined + ConvertFromAtoms. */
void orc_force(const orc_system *sys, orc_replica *rep);

/* Molecules::ExecuteStep<MODE>, src/integrator.cxx:646-706 (AoS variant). */
void orc_step(const orc_system *sys, orc_replica *rep);

/* Molecules::ExecuteSteps (src/integrator.cxx:708-803): nsteps steps then CalcProperties. */
void orc_execute_steps(const orc_system *sys, orc_replica *rep, int nsteps);

/* Molecules::CalcProperties, src/molecules.cxx:702-734. */
void orc_calc_properties(const orc_system *sys, orc_replica *rep);

/* REMDGPU::GetAverages field order (src/remdinfo.h:29-41, src/remdgpu.h:208-233):
 * LJ CLMB WALL VOL TRA ROT T P Px Py Pz TOT DRF TSTs TSTv BSTx BSTy BSTz DUMMY.
 * T and pressures are in reduced units (the REMDGPU convention). */
void orc_get_average(const orc_system *sys, const orc_replica *rep, double out[ORC_NUM_AVG]);

double orc_volume(const orc_system *sys, const orc_replica *rep);

/* Molecules::InitializeProperty (src/molecules.h:260-270). */
void orc_initialize_property(const orc_system *sys, orc_replica *rep);
/* Molecules::ChangeTemperature (src/molecules.h:333-353). */
void orc_change_temperature(const orc_system *sys, orc_replica *rep, double Tnew);
/* Molecules::KillMomentum (+ KillAngularMomentumInTube), src/molecules.cxx:168-210. */
void orc_kill_momentum(const orc_system *sys, orc_replica *rep);
/* Molecules::VelocityScaling / AngVelocityScaling, src/molecules.cxx:262-307. */
void orc_velocity_scaling(const orc_system *sys, orc_replica *rep);
void orc_ang_velocity_scaling(const orc_system *sys, orc_replica *rep);
/* The per-replica tail of REMD::ReplicaExchange for an exchanged replica
 * (src/remd.cxx:526-536): ChangeTemperature, KillMomentum, SetPressure,
 * CalcProperties, UpdateHamiltonian. */
void orc_apply_condition(const orc_system *sys, orc_replica *rep, double Tnew, double Pnew);

/* ---- exchange (src/remdinfo.cxx:54-125, 348-359; src/remd.cxx:467-538) ---- */
/* Pair lists: lists is 4 x (ntemp*npress/2) pairs {a,b}; returns lengths in len[4]. */
void orc_exchange_lists(int ntemp, int npress, int *lists, int len[4]);
/* SetConditionGeometrical: T in K and P in Pa -> reduced arrays of ntemp*npress. */
void orc_conditions_geometrical(int ntemp, int npress, double tmin_K, double tmax_K,
                                double pmin_Pa, double pmax_Pa, double *T, double *P);
/* One REMD::ReplicaExchange over the list step%4.  index/temperature/pressure
 * are REMDInfo's arrays (index: condition slot -> replica; T/P: per replica).
 * pot/vol per replica.  u[i] is the uniform compared for pair i.  accepted[i]
 * receives 1/0 per pair.  Returns the number of pairs tried. */
int orc_replica_exchange(int ntemp, int npress, int pconstant, long step,
                         int *index, double *temperature, double *pressure,
                         const double *pot, const double *vol, const double *u,
                         int *accepted, unsigned char *is_exchanged);

#ifdef __cplusplus
}
#endif
#endif
