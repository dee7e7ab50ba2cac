// device_state.cuh -- HBM layout of the B200 carrier engine: band tables,
// mesh / cell data, particle store and tallies, as seen by the kernels.
//
// All pointers are device pointers owned by the engine context (engine.cu).
// Structures are passed to kernels by value (kernel parameter space).
#pragma once

#include <cstdint>

namespace mcb200 {

constexpr int kNT = 7501;       // energy-table points (MTAB + 1)
constexpr int kMNB = 8;         // band slots
constexpr int kMWLE = 325;      // coarse tetrahedron-list bins (40 meV)
constexpr int kMWLES = 60;      // fine tetrahedron-list bins (2 meV)
constexpr int kMaxContacts = 16;
constexpr int kMaxSurfaces = 30;
constexpr int kSeedGridN = 96;  // cells per axis of the lowest-band walk-seed grid
// `step` word of the random stream used for initial-ensemble sampling.
constexpr uint32_t kSeedStreamStep = 0xfffffffdu;

// Motion rules (ldg actions), include/Constant_GlobalVariable_MathFunction.h:229-243.
enum MotionRule : int { kPass = 1, kReflect = 2, kScattOx = 3, kPeriod = 4, kGenerate = 5, kCatch = 6, kCatchGate = 7, kGenRef = 8 };
// Face directions, same header :204.
enum Dir : int { kUp = 0, kDown = 1, kLeft = 2, kRight = 3, kFront = 4, kBack = 5 };

// Full-band tables in device memory.  Everything the free flight reads about
// a tetrahedron on an event (face planes, velocity, neighbours, majorant,
// energy span, band) is packed into one record: one 128-byte L2 line in
// FP32, two in FP64 (55320 tets: 7 MB / 14 MB, L2-resident on B200).  R is the
// arithmetic type of the flight kinematics: double for the plain path,
// float for the FP32-flight path.
template <typename R>
struct TetFlightT {
  R n[4][4];    // face f: inward normal (n[f][0..2]) and offset n[f][3]
  R v[4];       // group velocity (v[0..2]) and base energy v[3]
  int neib[4];  // NeibrTet per face (>= 0 tet, < 0 wedge / BZ code)
  R gam;        // gamtet: the variable-gamma phonon majorant
  R e0, e3;     // lowest and highest node energy
  int band;     // ibt
  int node0;    // the first (lowest) node, the base of GetEnergy
  int pad[sizeof(R) == 4 ? 3 : 12];  // one 128-byte line (FP32) / two (FP64)
};
template <typename R>
struct TetShapeT {
  R e[4];     // node energies, ascending
  R fac[3];   // FASTSURF coefficients (low, medium, high)
  R vgt;      // |v|
};
using TetFlight = TetFlightT<double>;
using TetShape = TetShapeT<double>;

// FP32 copies of the tables the FP32 flight reads (built from the FP64
// tables by rounding each entry once).
struct DevTables32 {
  const TetFlightT<float> *tf;
  const TetShapeT<float> *ts;
  const float4 *knode;
  const float *gamtet, *energy, *sumscatt, *scatte, *dose, *scattiie, *scatth, *dosh, *scattiih, *dostetmax;
};

struct DevTables {
  int nt, nk, nbt;
  int nband[3], bandof[3];
  int scpre, scprh;
  double dtable, emax, dlist, dlists;
  double temptag, templag, templog, temptaf, templaf, temptof, temphop;
  double difpr[3];
  double mell, melt, meld;
  double a0pi, sieg, eV0, conc0, scrt0, eps_si, frickel;
  const TetFlight *tf;       // [nt]
  const TetShape *ts;        // [nt]
  const int4 *tnode;         // [nt] node indices
  const int4 *tneib;         // [nt] neighbour code per face
  const int *ibt;            // [nt]
  const double *gamtet;      // [nt]
  const double4 *knode;      // [nk] (kx, ky, kz, E)
  const double *energy;      // [kNT]
  const double *sumscatt;    // [kNT][kMNB]
  const double *scatte;      // [14][4][4]
  const double *dose;        // [14][4][kNT]
  const double *scattiie;    // [4][4][kNT]
  const double *scatth;      // [4][3][3]
  const double *dosh;        // [4][3][kNT]
  const double *scattiih;    // [3][3][kNT]
  const double *dostetmax;   // [kMNB][kNT]
  const double *dos;         // [kMNB][kNT]  (initial-state sampling)
  const double *sumdos;      // [kNT][3]
  double dosmax[3];
  const int *ntlist, *ptlist, *tlist;     // [kMWLE][kMNB], list
  const int *nslist, *pslist, *slist;
  const int *ntlists, *ptlists, *tlists;  // [kMWLES][kMNB], list
  // k-space locator grid (engine-built): per band, a uniform grid over the
  // irreducible wedge's bounding box; each cell lists the band's tets whose
  // bounding box overlaps it, in descending tet order.
  int grid_n;                 // cells per axis
  double grid_lo[3], grid_inv[3];
  const int *grid_start;      // [kMNB][grid_n^3 + 1]
  const int *grid_tets;
  // seed grid of the lowest conduction band: kSeedGridN^3 cells over the
  // same box, each holding a starting tetrahedron for the mesh walk (-1: none)
  double seed_inv[3];
  const int *seed_grid;
  // symmetry (copied to shared memory by each block)
  const int *symi;            // [48*6] matsym[c][s] stored as s*6+c
  const int *newisym;         // [5][48]
  const double *bz;           // [3][5][48]  (xbz, ybz, zbz)
  const int *indmat;          // [729]
  const int *reflect_isym;    // [3][48]: isym after mirroring k_x / k_y / k_z
  // phonon dispersion tables (FullBandTables::dispersion; null when absent)
  const double *disp;
  int disp_off[6];
  DevTables32 f32;            // FP32 flight tables (null until a context selects FP32 flight)
};

// Mesh in the reference's normalised units; cell (i, j, k) has linear index
// (j * nx + i) * nz + k (C_LINDEX_GHOST_ONE with one rank, include/defs.h).
struct DevMesh {
  int nx, ny, nz;               // cells per axis
  const double *lx, *ly, *lz;   // node coordinates [n+1]
  const double *dx, *dy, *dz;   // cell widths [n]
  const float *dxf, *dyf, *dzf; // cell widths rounded to float (FP32 flight: cell-relative positions)
  const int *motion;            // [cells][6]
  const int *contact;           // [cells] attached contact, 1-based, 0 = none
  const int *in_surf;           // [cells]
  const int *nearest_surf;      // [cells]
  const double *efield;         // [cells][3] electron-felt field already times ChargeSign
  const double *hfield;         // [cells][3] hole-felt field already times ChargeSign
  const double *rho;            // [cells] screening density |q|/vol (compute_cell_charge)
  const double *da;             // [cells] ionised doping density
  const double *e_rough, *e_sphon, *h_rough, *h_sphon;  // [cells] surface rates
  // FP32 flight: per cell, (electron-felt field, bh_a), (hole-felt field,
  // bh_b), (bh_emax, bh_beta, bh_ecut, 0) -- the fields and the
  // Brooks-Herring factors in float, rebuilt before each FP32 step
  const float4 *cell32;         // [cells][3]
  int surface_dir[kMaxSurfaces];
  int surface_scatter;          // Flag_SurfaceScatter
  int surface_impurity;         // Flag_SurfaceImpurityScatter
  int heat;                     // flag_heat: phonon events deposit heat
  int quantum;                  // Flag_QuantumCorrection: LO / TO / LA final energies from the dispersion tables
};

// Particle store: structure of arrays, one entry per particle.  R = double:
// absolute positions, 80 bytes per particle.  R = float (FP32 flight):
// positions relative to the low corner of the particle's cell, 56 bytes.
// Energy and charge stay FP64 in both.
template <typename R>
struct DevParticlesT {
  R *x, *y, *z;
  R *kx, *ky, *kz;
  double *energy, *charge;
  uint32_t *cell;       // packed i | j << 10 | k << 20
  int32_t *itet;
  uint32_t *meta;       // isym | type << 8 | flags << 16
  uint32_t *uid;
};
using DevParticles = DevParticlesT<double>;
using DevParticles32 = DevParticlesT<float>;

// Bytes of one particle in the store.
template <typename R>
constexpr int particle_bytes() { return 6 * (int)sizeof(R) + 2 * 8 + 4 * 4; }

// Fixed-point scales of the order-independent int64 tallies.
constexpr double kChargeScale = 1099511627776.0;  // 2^40 per unit normalised charge
constexpr double kEnergyScale = 4294967296.0;     // 2^32 per kB*T

// Device tallies; sums are int64 fixed point so they do not depend on the
// order in which threads add (bit-reproducible from run to run).
struct DevTallies {
  unsigned long long *counters;  // see TallyCounter
  long long *contact;            // [kMaxContacts][6]: ngen, qgen, egen, ncatch, qcatch, ecatch
  long long *lcurrent;           // [ny + 1] charge
  long long *rcurrent;           // [ny + 1]
  long long *heat_e;             // [(nx+1)(ny+1)(nz+1)] energy*|q|, node layout (j*(nx+1)+i)*(nz+1)+k
  long long *heat_h;
};
enum TallyCounter : int {
  kCntPhonon = 0,      // sttt.phononScatter
  kCntImpurity = 1,    // sttt.impurityScatter
  kCntCaught = 2,      // catch_par_num
  kCntGenerated = 3,   // gen_par
  kCntEvents = 4,      // free-flight loop iterations
  kCntUnfinished = 5,  // PASS across the outer y boundary (reference would spin)
  kCntTooManyEvents = 6,
  kCntChildOverflow = 7,
  kCntNoTet = 8,       // Getisym found no tetrahedron (particle caught)
  kCntZeroTime = 9,    // FP32 flight: too many consecutive zero-length events (particle caught)
  kCntNumCounters = 16
};

// A copy made mid-step by GENERATE / GENREF, to be flown for the rest of the step.
template <typename R>
struct DevChildrenT {
  R *x, *y, *z, *kx, *ky, *kz;
  double *energy, *charge, *left_time;
  uint32_t *cell;
  int32_t *itet;
  uint32_t *meta;
  uint32_t *parent_uid, *sub;
  unsigned int *count;
  int capacity;
};
using DevChildren = DevChildrenT<double>;

// A particle count that lives in device memory: *a (+ *b), at most `max`
// (with neither pointer: `max` itself, a count the host knows).  Per-step
// kernels read their sizes through it, so the host never waits for a count
// between launches.
struct DevCount {
  const unsigned int *a = nullptr, *b = nullptr;
  int max = 0;
  __device__ __forceinline__ int get() const {
    if (!a && !b) return max;
    const unsigned long long v = (unsigned long long)(a ? *a : 0u) + (b ? *b : 0u);
    return (int)(v < (unsigned long long)max ? v : (unsigned long long)max);
  }
};

// The child generations of one step (one buffer per generation).
constexpr int kChildGenerations = 4;
template <typename R>
struct ChildSetT {
  DevChildrenT<R> g[kChildGenerations];
  // offset of generation `gen` in the concatenation and the total count
  __device__ __forceinline__ int offset(int gen, int *total) const {
    int off = 0, at = 0;
#pragma unroll
    for (int q = 0; q < kChildGenerations; ++q) {
      if (q == gen) at = off;
      off += min((int)*g[q].count, g[q].capacity);
    }
    if (total) *total = off;
    return at;
  }
};

inline __host__ __device__ uint32_t pack_cell(int i, int j, int k) {
  return (uint32_t)i | ((uint32_t)j << 10) | ((uint32_t)k << 20);
}

}  // namespace mcb200
