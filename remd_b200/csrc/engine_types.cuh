// engine_types.cuh -- device data layout of the B200 REMD engine.
//
// All replicas of all ensembles of one handle live in one set of arrays:
//   * molecule state, FP64 structure-of-arrays, component-major
//     (r[c*N + g], c = 0..2; v likewise; q, p, n with 4 components; f with 3),
//     g = global molecule index = RepConst::mol_off + local index;
//   * per-step force records ("pack"), rebuilt by the integrate kernel after
//     the positions move: FP32 form = {int32 x,y,z fixed-point centre of mass,
//     float site offsets R(q) b_k} padded to 16 B; FP64 form = {double box
//     fraction, double site offsets};
//   * full neighbour lists, uint16 local indices, column-major inside a force
//     tile so that the lanes of a warp read consecutive words;
//   * per-replica scalars (thermostat, barostat, box, H0, condition) in two
//     buffers that the integrate and force kernels ping-pong between;
//   * partial sums per 32 consecutive molecules of a replica (one warp),
//     written by one kernel and reduced in molecule order by every CTA of the
//     same replica in the next kernel (deterministic: a replica's result
//     depends neither on its batch mates nor on the tile size).
#pragma once
#include <cstdint>

namespace remd {

constexpr int kMaxSites = 5;
constexpr int kNumAvg = 19;
constexpr double kFix = 4294967296.0;          // 2^32: fixed-point box fraction
constexpr double kFixInv = 1.0 / 4294967296.0;

// Per-replica constants (read-only on the device).
struct RepConst {
  int nmol, mol_off;       // molecules; first global index
  int tile_off, ntile;     // force/integrate tiles [tile_off, tile_off+ntile)
  int warp_off, nwarp;     // 32-molecule partial-sum units [warp_off, warp_off+nwarp)
  int nsite, c0;           // sites; first charged site (charged sites are [c0, nsite))
  int confined, tconstant, pconstant;
  int nfwall, wall_off;    // wall table entries and offset into the table array
  int nbr_cap;             // neighbour list capacity per molecule
  int ens;                 // ensemble index
  int pack_stride;         // words (FP32) or doubles (FP64) per pack record
  long long pack_off;      // first record word/double of this replica
  long long nbr_off;       // first neighbour word of tile_off
  double dt, dthalf;
  double rc, rs, coef_sw;  // switching: coef_sw = 1/(rs-rc)^5
  double skin;
  double Q, W;
  double mass, I[3];
  double wall_dr;          // table spacing: wall_length/nfwall (tube) or half of it (slit)
  double wall_length_param;   // A, as read from .inp
  double bottom_area;      // GetBottomArea (tube)
  double slit_width;       // wall length in reduced units (slit volume)
  double body[kMaxSites][3];
  double qq[kMaxSites][kMaxSites];
  double sgm2, eps;        // O-O Lennard-Jones: ((s+s)/2)^2 and sqrt(e e)
  double site_reach;       // max |site - centre of mass| (A): per-site images matter
                           // once L_d < 2 (rc + 2 site_reach)
};

// Per-replica scalars (two copies, ping-pong).
struct RepState {
  double s, Ps, Pv[3], L[3];
  double H0, T, P, gkT;
};

// Integrate-kernel partials of 32 molecules.
struct Part1 {
  double sum_Pv[3];
  double sum_Ps;
  double disp;             // max |displacement since the list build| (A, build box)
  double pad[3];
};

// Force-kernel partials of 32 molecules (raw ordered-pair sums; consumers halve lj/clmb/vir).
struct Part2 {
  double lj, clmb, wall, vir[3];
  long long npairs;        // ordered pairs within rc
  double pad;
};

struct Tile {
  int rep, start, count, pad;   // replica, first local molecule, molecules in tile
};

// Cell lists of a replica (rebuilt with its neighbour lists): the periodic box
// cut into nx x ny x nz cells at least as wide as the list radius (a dimension
// with fewer than three such cells is not cut), molecules counting-sorted by
// cell.  cell_start holds kMaxCells + 1 offsets per replica.
constexpr int kMaxCells = 2048;
struct CellGrid {
  int nx, ny, nz;
  int rebuild;                  // the head's decision for this force step
};

// Everything a kernel needs, passed by value.
struct DevPtrs {
  int N;                         // total molecules
  int ntiles, nrep;
  const RepConst* rc;
  const Tile* tiles;
  const int* order;              // force-launch block -> tile, costliest first (NULL: identity)
  double *r, *v, *q, *p, *f, *n; // SoA, component-major, stride N
  void* pack;                    // FP32 words or FP64 doubles
  int4* ref_com;                 // fixed-point com at the last list build
  int4* com;                     // FP32 form: current fixed-point com (written with the pack)
  double* Lbuild;                // per tile, 3 doubles (NaN = list invalid)
  uint16_t* nbr;                 // neighbour lists (rcut + skin)
  uint16_t* nbt;                 // FP32 form: per-step lists of the pairs within rcut (same layout)
  int* nt_cnt;                   // FP32 form: per molecule, nfar | nnear << 16 in nbt
  int* nbr_cnt;                  // per molecule
  const double* wall;            // {f, U} pairs
  Part1* part1;
  Part2* part2;
  double* avg;                   // nrep * kNumAvg
  int* status;                   // per replica health word
  int* err;                      // global error word (bit flags)
  CellGrid* cgrid;               // per replica: grid and rebuild decision of this force step
  int* cell_start;               // per replica, kMaxCells + 1 offsets into cell_mol
  int4* cell_com;                // per molecule (global index space): centres sorted by cell, .w = local index
  const double* newT;            // conditions for the next interval (per replica)
  const double* newP;
  const int* changed;            // 1 = apply the exchange tail at the interval start
  int tile0;                     // first tile of a launch over a tile range (order == NULL)
  int rep0, nrep_l;              // replicas [rep0, rep0 + nrep_l) of a launch (per-replica kernels)
  int bm_win;                    // words per row of the list-rebuild bitmap (kernels.cu)
};

enum : int { kErrNbrOverflow = 1, kErrNonFinite = 2, kErrHistRange = 4 };

// (volume, potential) histogram of the replicas of one ensemble, one per
// condition slot (REMDInfo's Histogram, src/remdinfo.h:93-139): kHistBins x
// kHistBins counts, per bin the sum of the 19 Average fields, and per slot the
// occupied range {vmin, vmax, pmin, pmax, samples}.  hist == NULL: not kept.
constexpr int kHistBins = 500;   // NUM_VOL = NUM_POT, src/remdinfo.h:22-23
struct HistEns {
  int* hist;       // [slot][v][p]
  double* ave;     // [slot][v][p][kNumAvg]
  int* bounds;     // [slot][5]
  double emin, emax, de;   // kJ/mol per molecule
  double vmin, vmax, dv;   // A^3 per molecule
};

}  // namespace remd
