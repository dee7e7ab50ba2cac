// flight_physics.cuh -- per-particle full-band free flight on the device.
//
// One thread owns one particle for one time step and runs the reference's
// event loop (MeshQuantities::particle_fly, src/mcmodel.cpp:1874-2161) with
// every routine it calls restated as device code below.  Each routine cites
// the reference lines it follows.  Arithmetic is IEEE double in the
// reference's operand order and this code is compiled without FMA
// contraction, so with the same random draws (include/mcb200_rng.h) the
// discrete outcomes (tetrahedron, wedge, cell, event type, final state) are
// the reference's; only libm transcendentals (log, sin, cos, pow with a
// negative exponent) may differ from glibc by an ulp.
//
// Device-side differences from the reference, each deliberate:
//  * no process exit: conditions where the reference calls exit() or loops
//    forever set a counter in the tally block and end the particle's step;
//  * the free-flight loop is capped (kMaxEvents) instead of only printing
//    TOO_MANY_LOOPS (src/mcmodel.cpp:2156);
//  * surface-phonon mechanism choice uses drand = Random() * sum(rates): the
//    reference reads an uninitialised local there (src/ParSurfaceScatter.cpp:94,149);
//  * FP32 flight (R = float) runs the same event loop with float kinematics:
//    positions relative to the cell's low corner, k, velocities, fields,
//    event times and rate lookups in float; energy, charge and the
//    remaining step time stay double.  Its own random stream (four float
//    uniforms per Philox block, mcb200_uniform_f32) and a rounding-tolerant
//    event clock (a zero event time is taken as an event now, not as the
//    reference's "Tf < MY_ZERO" catch) make it statistically, not bitwise,
//    equal to the FP64 path;
//  * the tetrahedron search after an impurity event (Getisym,
//    src/ParticleUtils.cpp:395-625) walks the mesh from the current
//    tetrahedron through face neighbours, falling back to a uniform k-grid
//    lookup, instead of scanning the reference's lists; both return the
//    tetrahedron of the band that contains k (they could differ only for a
//    k within 1e-13 of a face shared by two tetrahedra).
#pragma once

#include "device_state.cuh"
#include "mcb200_rng.h"

namespace mcb200 {

constexpr double kMyZero = 1e-13;          // MY_ZERO, include/defs.h
constexpr double kPiD = 3.141592653589793238462643e0;
constexpr int kMaxEvents = 1000000;
// FP32 flight: consecutive zero-length events after which a particle is
// taken as stuck (counted in kCntZeroTime and caught).
constexpr int kMaxZeroTimeEvents = 64;
// Opt-in event census (build with -DMCB200_FLIGHT_EVENT_STATS=1): counters
// 10-15 of the tallies count the flight loop's passes by the event that
// ended them and the work of the rare shared tails, for the design record
// (mcb200.flight_events); one atomic per counted event, so never in a
// timed build.
#ifndef MCB200_FLIGHT_EVENT_STATS
#define MCB200_FLIGHT_EVENT_STATS 0
#endif
enum EventStat : int {
  kStatTetFace = 10,    // passes ended at a tetrahedron face
  kStatCellFace = 11,   // at a cell face
  kStatScatter = 12,    // at a phonon, impurity or surface event (real or self-scattering)
  kStatStepEnd = 13,    // at the end of the step
  kStatStateTries = 14, // get_state draws (tetrahedra tried, accepted or not)
  kStatWalkSteps = 15,  // tetrahedra visited by the k-space walks
};

// Arithmetic of the two flight precisions.
template <typename R> struct FlightReal;
template <> struct FlightReal<double> {
  using V4 = double4;
  static constexpr bool kCellRelative = false;  // absolute positions, reference arithmetic
  static constexpr double kContain = kMyZero;   // face test d >= -kContain (unnormalised faces)
  static constexpr double kBig = 1e99;
};
template <> struct FlightReal<float> {
  using V4 = float4;
  static constexpr bool kCellRelative = true;   // positions relative to the cell's low corner
  static constexpr float kContain = 2e-5f;      // unit face normals: a k-space distance, ~10 float ulps at the BZ edge
  static constexpr float kBig = 1e30f;
};

__device__ __forceinline__ double m_abs(double v) { return fabs(v); }
__device__ __forceinline__ float m_abs(float v) { return fabsf(v); }
__device__ __forceinline__ double m_sqrt(double v) { return sqrt(v); }
__device__ __forceinline__ float m_sqrt(float v) { return sqrtf(v); }
__device__ __forceinline__ double m_log(double v) { return log(v); }
__device__ __forceinline__ float m_log(float v) { return logf(v); }
__device__ __forceinline__ double m_floor(double v) { return floor(v); }
__device__ __forceinline__ float m_floor(float v) { return floorf(v); }
__device__ __forceinline__ void m_sincos(double v, double *s, double *c) { *s = sin(v); *c = cos(v); }
__device__ __forceinline__ void m_sincos(float v, float *s, float *c) { sincosf(v, s, c); }

// Table views per precision (the FP64 tables or their FP32 copies).
template <typename R> struct Tab;
template <> struct Tab<double> {
  static __device__ __forceinline__ const TetFlightT<double> *tf(const DevTables &T) { return T.tf; }
  static __device__ __forceinline__ const TetShapeT<double> *ts(const DevTables &T) { return T.ts; }
  static __device__ __forceinline__ const double4 *knode(const DevTables &T) { return T.knode; }
  static __device__ __forceinline__ const double *gamtet(const DevTables &T) { return T.gamtet; }
  static __device__ __forceinline__ const double *energy(const DevTables &T) { return T.energy; }
  static __device__ __forceinline__ const double *sumscatt(const DevTables &T) { return T.sumscatt; }
  static __device__ __forceinline__ const double *scatte(const DevTables &T) { return T.scatte; }
  static __device__ __forceinline__ const double *dose(const DevTables &T) { return T.dose; }
  static __device__ __forceinline__ const double *scattiie(const DevTables &T) { return T.scattiie; }
  static __device__ __forceinline__ const double *scatth(const DevTables &T) { return T.scatth; }
  static __device__ __forceinline__ const double *dosh(const DevTables &T) { return T.dosh; }
  static __device__ __forceinline__ const double *scattiih(const DevTables &T) { return T.scattiih; }
  static __device__ __forceinline__ const double *dostetmax(const DevTables &T) { return T.dostetmax; }
};
template <> struct Tab<float> {
  static __device__ __forceinline__ const TetFlightT<float> *tf(const DevTables &T) { return T.f32.tf; }
  static __device__ __forceinline__ const TetShapeT<float> *ts(const DevTables &T) { return T.f32.ts; }
  static __device__ __forceinline__ const float4 *knode(const DevTables &T) { return T.f32.knode; }
  static __device__ __forceinline__ const float *gamtet(const DevTables &T) { return T.f32.gamtet; }
  static __device__ __forceinline__ const float *energy(const DevTables &T) { return T.f32.energy; }
  static __device__ __forceinline__ const float *sumscatt(const DevTables &T) { return T.f32.sumscatt; }
  static __device__ __forceinline__ const float *scatte(const DevTables &T) { return T.f32.scatte; }
  static __device__ __forceinline__ const float *dose(const DevTables &T) { return T.f32.dose; }
  static __device__ __forceinline__ const float *scattiie(const DevTables &T) { return T.f32.scattiie; }
  static __device__ __forceinline__ const float *scatth(const DevTables &T) { return T.f32.scatth; }
  static __device__ __forceinline__ const float *dosh(const DevTables &T) { return T.f32.dosh; }
  static __device__ __forceinline__ const float *scattiih(const DevTables &T) { return T.f32.scattiih; }
  static __device__ __forceinline__ const float *dostetmax(const DevTables &T) { return T.f32.dostetmax; }
};

// Symmetry tables staged in shared memory (one copy per block).
template <typename R>
struct SymSmemT {
  int symi[48 * 6];   // matsym[c][s] at s*6+c
  int newisym[5 * 48];
  R bz[3 * 5 * 48];
  int refl[3 * 48];
};
using SymSmem = SymSmemT<double>;

template <typename R>
struct FlightInstT {  // one simulation: its mesh and fields, tallies, copy buffer and step
  DevMesh M;
  DevTallies Y;
  DevChildrenT<R> C;
  double dt;
  uint64_t seed;
  uint32_t step;
  // when set, the step number is read here on the device instead (launches
  // captured in a CUDA graph and replayed at later steps)
  const uint32_t *step_dev = nullptr;
};
template <typename R>
struct FlightCtxT : FlightInstT<R> {  // plus the band tables, shared by every simulation
  DevTables T;
};

// One simulation of a batched flight launch: its flight context, its
// current particle store and device count (main flight), or the copies it
// flies (child flights).
template <typename R>
struct BatchInstT : FlightInstT<R> {
  DevParticlesT<R> P;
  DevChildrenT<R> in;
  const unsigned int *n;
  int capacity;
  int pad_;
};
constexpr int kMaxBatch = 64;  // simulations per batched launch (their table fits in shared memory)
using FlightCtx = FlightCtxT<double>;

__device__ __forceinline__ void tally_add_i64(long long *p, double v, double scale) {
  atomicAdd(reinterpret_cast<unsigned long long *>(p), (unsigned long long)__double2ll_rn(v * scale));
}
__device__ __forceinline__ void count(const DevTallies &Y, int which) { atomicAdd(&Y.counters[which], 1ull); }

template <typename R>
struct FlyerT {
  using Real = FlightReal<R>;
  using V4 = typename Real::V4;
  using TB = Tab<R>;
  const FlightCtxT<R> &F;      // the tables (F.T)
  const SymSmemT<R> &S;
  const FlightInstT<R> *I;     // the simulation of the current particle (F itself unless batched)
  // random stream (uid, step_, sub; step_ set by the launch's IO from the
  // simulation's step) and the cached Philox block (index rblk, words rw0..rw3)
  uint32_t uid, sub, n, step_;
  uint32_t rblk, rw0, rw1, rw2, rw3;
  // particle registers (MeshQuantities members, include/mcmodel.h:215-233)
  R x, y, z, kx, ky, kz;
  double energy, charge, left_time;
  int ic, jc, kc, itet, isym, type, iband;
  R Ex, Ey, Ez, vx, vy, vz;
  double Rho, DA;                                // FP64: cell screening and doping densities
  R imp_a, imp_b, imp_ecut, imp_emax, imp_beta;  // FP32: the cell's Brooks-Herring constants
  int itetdir, idir;
  bool catch_, self;
  R rough_rate, sphon_rate, surf_gamma, imp_gamma;
  int nchild;
  // Work left by an event handler for the shared tails of the event loop
  // (one call site each for the mechanism search, the final-state draw and
  // the k-point search; see run_pick / run_final_state / run_locate).
  bool pick_pending;
  R pick_drand;
  int fs_kind, fs_tal;  // pending final-state draw: kind and wedge rule
  double fs_eeold;      // state before the draw (restored on self-scattering)
  R fs_kx, fs_ky, fs_kz;
  int fs_ib, fs_it, fs_is;
  int loc_mode;         // pending k-point search
  enum : int { kFsNone = 0, kFsPhonon = 1, kFsIonize = 2, kFsDiffuse = 3 };
  enum : int { kLocNone = 0, kLocBZ = 1, kLocImpurity = 2 };

  __device__ FlyerT(const FlightCtxT<R> &f, const SymSmemT<R> &s) : F(f), S(s), I(&f), step_(f.step) {}

  __device__ __forceinline__ void start_stream(uint32_t u, uint32_t sb) {
    uid = u;
    sub = sb;
    n = 0;
    rblk = 0xffffffffu;
  }

  // Draw n of the particle's stream (include/mcb200_rng.h).  FP64: the
  // 52-bit uniforms of mcb200_uniform, two per Philox block; FP32: the
  // 23-bit uniforms of mcb200_uniform_f32, four per block.  A block is
  // computed once and kept for the draws that follow.
  __device__ __forceinline__ R Random() {
    if constexpr (sizeof(R) == 8) {
      const uint32_t b = n >> 1;
      double u;
      if ((n & 1u) && b == rblk) {
        u = mcb200_bits_to_unit(rw3, rw2);
      } else {
        const mcb200_philox_block w =
            mcb200_philox4x32_10(b, uid, step_, sub, (uint32_t)I->seed, (uint32_t)(I->seed >> 32));
        rblk = b;
        rw2 = w.w[2];
        rw3 = w.w[3];
        u = (n & 1u) ? mcb200_bits_to_unit(w.w[3], w.w[2]) : mcb200_bits_to_unit(w.w[1], w.w[0]);
      }
      ++n;
      return u;
    } else {
      const uint32_t b = n >> 2;
      if (b != rblk) {
        const mcb200_philox_block w =
            mcb200_philox4x32_10(b, uid, step_, sub, (uint32_t)I->seed, (uint32_t)(I->seed >> 32));
        rblk = b;
        rw0 = w.w[0];
        rw1 = w.w[1];
        rw2 = w.w[2];
        rw3 = w.w[3];
      }
      const uint32_t q = n & 3u;
      const uint32_t w = q == 0 ? rw0 : (q == 1 ? rw1 : (q == 2 ? rw2 : rw3));
      ++n;
      return mcb200_bits_to_unit_f32(w);
    }
  }

  __device__ __forceinline__ int ms(int c, int s) const { return S.symi[s * 6 + c]; }
  __device__ __forceinline__ int cell_index() const { return (jc * I->M.nx + ic) * I->M.nz + kc; }
  __device__ __forceinline__ int cell_index(int i, int j, int k) const { return (j * I->M.nx + i) * I->M.nz + k; }
  __device__ __forceinline__ const TetFlightT<R> &tf(int it) const { return TB::tf(F.T)[it]; }
  __device__ __forceinline__ const TetShapeT<R> &ts(int it) const { return TB::ts(F.T)[it]; }

  // in_wedge, src/ParticleUtils.cpp:295-305: BZ vector -> irreducible wedge of isym.
  __device__ __forceinline__ void in_wedge(R &xo, R &yo, R &zo, R xi, R yi, R zi) const {
    const int p0 = ms(0, isym) - 1, p1 = ms(1, isym) - 1;
    const R a = xi * (R)ms(3, isym), b = yi * (R)ms(4, isym), c = zi * (R)ms(5, isym);
    xo = p0 == 0 ? a : (p1 == 0 ? b : c);
    yo = p0 == 1 ? a : (p1 == 1 ? b : c);
    zo = p0 == 2 ? a : (p1 == 2 ? b : c);
  }
  // Band::OutWedge, src/Band.cpp:555-570: wedge vector -> BZ.
  __device__ __forceinline__ void out_wedge(R &xo, R &yo, R &zo, R xi, R yi, R zi) const {
    const int p0 = ms(0, isym) - 1, p1 = ms(1, isym) - 1, p2 = ms(2, isym) - 1;
    xo = (p0 == 0 ? xi : (p0 == 1 ? yi : zi)) * (R)ms(3, isym);
    yo = (p1 == 0 ? xi : (p1 == 1 ? yi : zi)) * (R)ms(4, isym);
    zo = (p2 == 0 ? xi : (p2 == 1 ? yi : zi)) * (R)ms(5, isym);
  }
  // GetV, src/ParticleUtils.cpp:307-313.
  __device__ __forceinline__ void GetV() {
    const V4 v = *reinterpret_cast<const V4 *>(tf(itet).v);
    out_wedge(vx, vy, vz, v.x, v.y, v.z);
  }
  // GetEnergy, src/ParticleUtils.cpp:315-329.
  __device__ void GetEnergy() {
    R dx, dy, dz;
    in_wedge(dx, dy, dz, kx, ky, kz);
    const TetFlightT<R> &t = tf(itet);
    const V4 k0 = TB::knode(F.T)[t.node0];
    dx -= k0.x;
    dy -= k0.y;
    dz -= k0.z;
    const R *v = t.v;
    energy = v[3] + v[0] * dx + v[1] * dy + v[2] * dz;
  }
  __device__ __forceinline__ R face_dist(int it, int f, R a, R b, R c) const {
    const R *nn = tf(it).n[f];
    return nn[0] * a + nn[1] * b + nn[2] * c - nn[3];
  }
  __device__ __forceinline__ bool tet_contains(int it, R a, R b, R c) const {
    const R tol = -Real::kContain;
    return face_dist(it, 0, a, b, c) >= tol && face_dist(it, 1, a, b, c) >= tol &&
           face_dist(it, 2, a, b, c) >= tol && face_dist(it, 3, a, b, c) >= tol;
  }

  // TetTime, src/TetHit.cpp:4-106: time to the tet face the drift reaches first.
  __device__ R TetTime() {
    R xkl, ykl, zkl, xfl, yfl, zfl;
    in_wedge(xkl, ykl, zkl, kx, ky, kz);
    in_wedge(xfl, yfl, zfl, Ex, Ey, Ez);
    const TetFlightT<R> &t = tf(itet);
    R best = 0;
    itetdir = 0;
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      const R nf = t.n[f][0] * xfl + t.n[f][1] * yfl + t.n[f][2] * zfl;
      R tfp;
      if (nf < 0) {
        tfp = (t.n[f][3] - (t.n[f][0] * xkl + t.n[f][1] * ykl + t.n[f][2] * zkl)) / nf;
        if (tfp < 0) tfp = 0;
      } else {
        tfp = Real::kBig;
      }
      if (f == 0) best = tfp;
      else if (tfp < best) {
        best = tfp;
        itetdir = f;
      }
    }
    return best;
  }

  // CellTime, src/CellHit.cpp:4-93: time to the real-space cell face.  FP32
  // positions are offsets from the cell's low corner, so the gaps are
  // (width - x) and x.
  __device__ R CellTime() {
    const DevMesh &M = I->M;
    int idx, idy, idz;
    R tx, ty, tz;
    if constexpr (Real::kCellRelative) {
      if (vx > 0) { idx = kDown; tx = (M.dxf[ic] - x) / vx; }
      else if (vx < 0) { idx = kUp; tx = -x / vx; }
      else { idx = kUp; tx = Real::kBig; }
      if (vy > 0) { idy = kRight; ty = (M.dyf[jc] - y) / vy; }
      else if (vy < 0) { idy = kLeft; ty = -y / vy; }
      else { idy = kRight; ty = Real::kBig; }
      if (vz > 0) { idz = kBack; tz = (M.dzf[kc] - z) / vz; }
      else if (vz < 0) { idz = kFront; tz = -z / vz; }
      else { idz = kFront; tz = Real::kBig; }
    } else {
      if (vx > 0) { idx = kDown; tx = (M.lx[ic + 1] - x) / vx; }
      else if (vx < 0) { idx = kUp; tx = -(x - M.lx[ic]) / vx; }
      else { idx = kUp; tx = Real::kBig; }
      if (vy > 0) { idy = kRight; ty = (M.ly[jc + 1] - y) / vy; }
      else if (vy < 0) { idy = kLeft; ty = -(y - M.ly[jc]) / vy; }
      else { idy = kRight; ty = Real::kBig; }
      if (vz > 0) { idz = kBack; tz = (M.lz[kc + 1] - z) / vz; }
      else if (vz < 0) { idz = kFront; tz = -(z - M.lz[kc]) / vz; }
      else { idz = kFront; tz = Real::kBig; }
    }
    idir = idx;
    R t = tx;
    if (ty < t) { idir = idy; t = ty; }
    if (tz < t) { idir = idz; t = tz; }
    if constexpr (Real::kCellRelative) {
      if (t < 0) t = 0;  // a position rounded just past the face
    } else {
      if (t < -kMyZero) t = 0;
    }
    return t;
  }

  // Band::CONFBZ, src/Band.cpp:573-616: fold k back into the first BZ.
  __device__ void CONFBZ(R &a, R &b, R &c) const {
    const R p = (R)F.T.a0pi;
    for (int guard = 0; guard < 64; ++guard) {
      bool out = m_abs(a) > p || m_abs(b) > p || m_abs(c) > p || m_abs(a) + m_abs(b) + m_abs(c) > (R)1.50 * p;
      if (!out) return;
      a = a > (R)0 ? a - p : a + p;
      b = b > (R)0 ? b - p : b + p;
      c = c > (R)0 ? c - p : c + p;
    }
  }

  // Point location by walking the tetrahedral mesh: from `start`, repeatedly
  // step through the face whose plane the point lies furthest outside of,
  // until every face test passes (the reference's containment test,
  // d >= -MY_ZERO).  Returns -1 when the walk reaches a wedge boundary or
  // does not settle within the step cap; the caller then uses the k-grid.
  __device__ int walk_to(int start, R a, R b, R c) const {
    int it = start;
    for (int s = 0; s < 64; ++s) {
      if constexpr (MCB200_FLIGHT_EVENT_STATS != 0) count(I->Y, kStatWalkSteps);
      int fmin = -1;
      R dmin = -Real::kContain;
#pragma unroll
      for (int f = 0; f < 4; ++f) {
        const R d = face_dist(it, f, a, b, c);
        if (d < dmin) {
          dmin = d;
          fmin = f;
        }
      }
      if (fmin < 0) return it;
      const int nb = tf(it).neib[fmin];
      if (nb < 0) return -1;
      it = nb;
    }
    return -1;
  }

  // Getisym, src/ParticleUtils.cpp:395-625: wedge from k, then the tet of
  // band iband that contains the wedge vector (k-grid lookup, see file note).
  __device__ void Getisym() {
    int mink, maxk;
    R tmin, tmax;
    if (m_abs(kx) > m_abs(ky)) { tmin = m_abs(ky); tmax = m_abs(kx); mink = 1; maxk = 0; }
    else { tmin = m_abs(kx); tmax = m_abs(ky); mink = 0; maxk = 1; }
    if (m_abs(kz) < tmin) mink = 2;
    else if (m_abs(kz) > tmax) maxk = 2;
    // pos[mink] = 2, pos[maxk] = 0, else 1 (mink != maxk always)
    const int p0 = maxk == 0 ? 0 : (mink == 0 ? 2 : 1);
    const int p1 = maxk == 1 ? 0 : (mink == 1 ? 2 : 1);
    const int p2 = maxk == 2 ? 0 : (mink == 2 ? 2 : 1);
    int sx, sy, sz;
    if constexpr (sizeof(R) == 8) {
      auto sgn = [](double v) { return (int)(fabs(v) / v); };  // utils.cpp sign()
      sx = sgn(kx) + 1; sy = sgn(ky) + 1; sz = sgn(kz) + 1;
    } else {
      // a component rounded to exactly zero lies on a wedge plane: either
      // side's wedge contains it, take the positive one
      sx = kx < 0 ? 0 : 2; sy = ky < 0 ? 0 : 2; sz = kz < 0 ? 0 : 2;
    }
    if (sx < 0 || sx > 2 || sy < 0 || sy > 2 || sz < 0 || sz > 2) {  // a zero component: sign() is NaN in the reference
      count(I->Y, kCntNoTet);
      catch_ = true;
      return;
    }
    isym = F.T.indmat[((((sx * 3 + sy) * 3 + sz) * 3 + p0) * 3 + p1) * 3 + p2];
    R a, b, c;
    in_wedge(a, b, c, kx, ky, kz);
    const bool same_band = iband == tf(itet).band;
    if (same_band && tet_contains(itet, a, b, c)) return;
    int start = same_band ? itet : -1;
    if (iband == F.T.bandof[0]) {  // lowest conduction band: start next to the point
      const int sg = kSeedGridN;
      const int si = min(max((int)m_floor((a - (R)F.T.grid_lo[0]) * (R)F.T.seed_inv[0]), 0), sg - 1);
      const int sj = min(max((int)m_floor((b - (R)F.T.grid_lo[1]) * (R)F.T.seed_inv[1]), 0), sg - 1);
      const int sk = min(max((int)m_floor((c - (R)F.T.grid_lo[2]) * (R)F.T.seed_inv[2]), 0), sg - 1);
      const int s0 = F.T.seed_grid[((size_t)si * sg + sj) * sg + sk];
      if (s0 >= 0) start = s0;
    }
    if (start >= 0) {
      const int w = walk_to(start, a, b, c);
      if (w >= 0) {
        itet = w;
        return;
      }
    }
    const int g = F.T.grid_n;
    int gi = (int)m_floor((a - (R)F.T.grid_lo[0]) * (R)F.T.grid_inv[0]);
    int gj = (int)m_floor((b - (R)F.T.grid_lo[1]) * (R)F.T.grid_inv[1]);
    int gk = (int)m_floor((c - (R)F.T.grid_lo[2]) * (R)F.T.grid_inv[2]);
    gi = min(max(gi, 0), g - 1);
    gj = min(max(gj, 0), g - 1);
    gk = min(max(gk, 0), g - 1);
    const int *st = F.T.grid_start + (size_t)iband * (g * g * g + 1);
    const int cell = (gi * g + gj) * g + gk;
    for (int q = st[cell]; q < st[cell + 1]; ++q) {
      const int it = F.T.grid_tets[q];
      if (tet_contains(it, a, b, c)) {
        itet = it;
        return;
      }
    }
    count(I->Y, kCntNoTet);
    catch_ = true;
  }

  // GetisymBZ, src/ParticleUtils.cpp:331-392, first part: after a
  // BZ-boundary crossing, the current tet or one of the BZ-surface tets of
  // the particle's energy bin; false leaves the search to Getisym.
  __device__ bool bz_surface_search() {
    R a, b, c;
    in_wedge(a, b, c, kx, ky, kz);
    if (iband == tf(itet).band && tet_contains(itet, a, b, c)) return true;
    int ie = (int)(energy * F.T.dlist);
    if (ie < 0) ie = 0;
    if (ie >= kMWLE) ie = kMWLE - 1;
    const int p = F.T.pslist[ie * kMNB + iband], cnt = F.T.nslist[ie * kMNB + iband];
    for (int itl = p; itl <= p + cnt - 1; ++itl) {
      const int it = F.T.slist[itl];
      if (iband == tf(it).band && tet_contains(it, a, b, c)) {
        itet = it;
        return true;
      }
    }
    return false;
  }

  // HitTet, src/TetHit.cpp:109-142.  After a BZ-boundary crossing the tet
  // search and GetEnergy run in run_locate.
  __device__ void HitTet() {
    const int nb = tf(itet).neib[itetdir];
    if (nb >= 0) {
      itet = nb;
    } else if (nb == -5 || nb == -6) {
      const int ii = -nb - 2;
      kx = kx + S.bz[(0 * 5 + ii) * 48 + isym];
      ky = ky + S.bz[(1 * 5 + ii) * 48 + isym];
      kz = kz + S.bz[(2 * 5 + ii) * 48 + isym];
      isym = S.newisym[ii * 48 + isym];
      loc_mode = kLocBZ;
    } else {
      isym = S.newisym[(-nb - 2) * 48 + isym];
    }
  }

  // The k-point search after a BZ crossing (GetisymBZ, then GetEnergy unless
  // the particle was caught: src/TetHit.cpp:129-134) or after an accepted
  // impurity event (Getisym, then GetEnergy:
  // src/ElectronImpurityScatter.cpp:291-296).
  __device__ void run_locate() {
    const bool bz = loc_mode == kLocBZ;
    loc_mode = kLocNone;
    if (!(bz && bz_surface_search())) Getisym();
    if (bz && catch_) return;
    GetEnergy();
  }

  // TALIND, src/ParticleUtils.cpp:626-748: final valley (and a random wedge
  // in it).  The reference's talend[] lookups are written as arithmetic on
  // the drawn index (1..4); an index of 5 (u*4+1 rounding up to 5, possible
  // only for u within 2^-51 of 1) reads past the reference's table and is
  // clamped to 4 here.
  __device__ __forceinline__ int talend_index() { return min((int)(Random() * (R)4.0 + (R)1.0), 4); }
  __device__ void TALIND(int ityp) {
    int ital = 1;
    const R ax = m_abs(kx), ay = m_abs(ky), az = m_abs(kz);
    if (ax >= ay && ax >= az) {
      if (kx >= (R)0) {
        if (ityp == 1) ital = 1;
        if (ityp == 2) ital = 2;
        if (ityp == 3) ital = talend_index() + 2;  // {3,4,5,6}
      }
      if (kx < (R)0) {
        if (ityp == 1) ital = 2;
        if (ityp == 2) ital = 1;
        if (ityp == 3) ital = talend_index() + 2;
      }
    }
    if (ay >= az && ay >= ax) {
      if (ky >= (R)0) {
        if (ityp == 1) ital = 3;
        if (ityp == 2) ital = 4;
        if (ityp == 3) { const int i = talend_index(); ital = i <= 2 ? i : i + 2; }  // {1,2,5,6}
      }
      if (ky < (R)0) {
        if (ityp == 1) ital = 4;
        if (ityp == 2) ital = 3;
        if (ityp == 3) { const int i = talend_index(); ital = i <= 2 ? i : i + 2; }
      }
    }
    if (az > ay && az > ax) {
      if (kz >= (R)0) {
        if (ityp == 1) ital = 5;
        if (ityp == 2) ital = 6;
        if (ityp == 3) ital = talend_index();  // {1,2,3,4}
      }
      if (kz < (R)0) {
        if (ityp == 1) ital = 6;
        if (ityp == 2) ital = 5;
        if (ityp == 3) ital = talend_index();
      }
    }
    isym = (int)(Random() * (R)8.0) + 8 * (ital - 1);
  }

  // Band::CALDOSTETMAX, src/Band.cpp:2298-2320.
  __device__ R CALDOSTETMAX(R eed, int ib) const {
    const R *d = TB::dostetmax(F.T) + (size_t)ib * kNT;
    if (eed <= (R)0) return d[0];
    if (eed >= (R)F.T.emax) return d[kNT - 1];
    const int itab = min((int)(eed / (R)F.T.dtable), kNT - 2);  // eed just below emax may round to the last point
    return d[itab] > d[itab + 1] ? d[itab] : d[itab + 1];
  }

  // Band::SURF, src/Band.cpp:194-332 (only reached by FASTSURF for
  // tetrahedra whose two lowest nodes are degenerate).
  __device__ R SURF(R eps, int it) const;
  // Band::FASTSURF, src/Band.cpp:665-704.
  __device__ R FASTSURF(R eps, int it) const {
    const TetShapeT<R> &s = ts(it);
    const R e0 = s.e[0], e1 = s.e[1], e2 = s.e[2], e3 = s.e[3];
    if (eps > e0 && eps < e3) {
      if (eps <= e1) return s.fac[0] * (eps - e0) * (eps - e0);
      if (eps < e2) {
        if (e1 - e0 > (R)1e-10) return s.fac[0] * (eps - e0) * (eps - e0) - s.fac[1] * (eps - e1) * (eps - e1);
        return SURF(eps, it);
      }
      return s.fac[2] * (eps - e3) * (eps - e3);
    }
    return 0;
  }

  // get_state, src/ParticleUtils.cpp:48-120: random final state on the
  // iso-energy surface of band iband (rejection on the tet's DOS share).
  __device__ void get_state() {
    if (energy <= 0.0) {
      self = true;
      return;
    }
    const R e = (R)energy;
    const R maxdostet = CALDOSTETMAX(e, iband);
    int itab = (int)(e * (R)F.T.dlists);
    bool small_ = itab < kMWLES;
    if (!small_) {
      itab = (int)(e * (R)F.T.dlist);
      if (itab >= kMWLE) itab = kMWLE - 1;
    }
    const int nted = small_ ? F.T.ntlists[itab * kMNB + iband] : F.T.ntlist[itab * kMNB + iband];
    const int base = small_ ? F.T.ptlists[itab * kMNB + iband] : F.T.ptlist[itab * kMNB + iband];
    const int *lst = small_ ? F.T.tlists : F.T.tlist;
    if (nted == 0) {
      self = true;
      return;
    }
    int count2 = 0;
    for (;;) {
      int pick = (int)(nted * Random());
      if constexpr (sizeof(R) == 4) pick = min(pick, nted - 1);
      itet = lst[pick + base];
      count2++;
      const TetShapeT<R> &s = ts(itet);
      if ((count2 < 10000) && !((s.e[0] < e) && (s.e[3] > e))) continue;
      const R dostet = FASTSURF(e, itet) / s.vgt;
      if (((Random() * maxdostet) > dostet) && (count2 < 10000)) continue;
      break;
    }
    if constexpr (MCB200_FLIGHT_EVENT_STATS != 0)
      atomicAdd(&I->Y.counters[kStatStateTries], (unsigned long long)count2);
    if (count2 >= 10000) {
      self = true;
    } else {
      self = false;
      getK();
    }
  }

  // getK, src/ParticleUtils.cpp:122-284: uniform point on the iso-energy
  // triangle / quadrangle of tet itet, mapped out of the wedge.
  __device__ void getK();

  // Band::CALSCATTSUM, src/Band.cpp:1999-2033.
  __device__ R CALSCATTSUM(R eed, int ib) const {
    const R *s = TB::sumscatt(F.T);
    const R *E = TB::energy(F.T);
    if (eed <= (R)0) return s[ib];
    if (eed >= (R)F.T.emax) return s[(size_t)(kNT - 1) * kMNB + ib];
    const int itab = min((int)(eed / (R)F.T.dtable), kNT - 2);
    const R intp = (eed - E[itab]) / (E[itab + 1] - E[itab]);
    return s[(size_t)itab * kMNB + ib] + intp * (s[(size_t)(itab + 1) * kMNB + ib] - s[(size_t)itab * kMNB + ib]);
  }

  // Electron mechanism choice by a running sum over Band::CALSCATTE
  // (src/Band.cpp:2165-2231) entries, without materialising the 56-entry
  // array: returns the chosen index or -1 (self-scattering).
  __device__ int pick_electron_mechanism(R drand) const;
  __device__ R electron_rate_sum() const;
  __device__ int pick_hole_mechanism(R drand) const;
  __device__ R hole_rate_sum() const;

  // heat_to_point, src/heat.cpp:169-196 (CIC onto the cell's 8 nodes).
  __device__ void heat_to_point(double e, long long *heat) const {
    const DevMesh &M = I->M;
    R rx, ry, rz;
    if constexpr (Real::kCellRelative) {
      rx = x / M.dxf[ic];
      ry = y / M.dyf[jc];
      rz = z / M.dzf[kc];
    } else {
      rx = (x - M.lx[ic]) / M.dx[ic];
      ry = (y - M.ly[jc]) / M.dy[jc];
      rz = (z - M.lz[kc]) / M.dz[kc];
    }
    const int px = M.nx + 1, pz = M.nz + 1;
    auto node = [&](int i, int j, int k) { return ((size_t)j * px + i) * pz + k; };
    tally_add_i64(heat + node(ic, jc, kc), e * (1 - ry) * (1 - rx) * (1 - rz), kEnergyScale);
    tally_add_i64(heat + node(ic + 1, jc, kc), e * (1 - ry) * rx * (1 - rz), kEnergyScale);
    tally_add_i64(heat + node(ic, jc, kc + 1), e * (1 - ry) * (1 - rx) * rz, kEnergyScale);
    tally_add_i64(heat + node(ic + 1, jc, kc + 1), e * (1 - ry) * rx * rz, kEnergyScale);
    tally_add_i64(heat + node(ic, jc + 1, kc), e * ry * (1 - rx) * (1 - rz), kEnergyScale);
    tally_add_i64(heat + node(ic + 1, jc + 1, kc), e * ry * rx * (1 - rz), kEnergyScale);
    tally_add_i64(heat + node(ic, jc + 1, kc + 1), e * ry * (1 - rx) * rz, kEnergyScale);
    tally_add_i64(heat + node(ic + 1, jc + 1, kc + 1), e * ry * rx * rz, kEnergyScale);
  }

  // ---- final states ----------------------------------------------------
  // The reference draws a final state inside EPSCAT / ESCATII (electrons),
  // HPSCAT / HSCATII (holes) and Diffuse.  Here the event handlers set up the
  // mechanism's band, energy and wedge rule (request_scatter,
  // request_diffuse) and one shared tail, run_final_state, makes the draws
  // in the reference's order (the wedge: TALIND or a random isym; then
  // get_state) and applies the routine's epilogue.  One call site of
  // get_state / TALIND / getK keeps the event loop small enough for the
  // instruction cache.
  __device__ void save_old() {
    fs_eeold = energy;
    fs_kx = kx; fs_ky = ky; fs_kz = kz;
    fs_ib = iband; fs_it = itet; fs_is = isym;
  }
  __device__ void restore_k() {
    kx = fs_kx; ky = fs_ky; kz = fs_kz;
    iband = fs_ib; itet = fs_it; isym = fs_is;
  }

  // FEKLOEM / FEKLOAB / FEKTOEM / FEKTOAB / FEKLAEM / FEKLAAB
  // (src/ElectronPhononScatter.cpp:633-1022), table-driven: the final energy
  // of an LO / TO / LA phonon event under quantum correction.  The energy in
  // phonon quanta selects a column of the dispersion table (per-range
  // offset, scale and spacing edeta); one draw walks the column's
  // cumulative sum to a row i, and the final energy is the phonon energy
  // shifted by +-(i / 2) steps of c * edeta.  Below one quantum the emission
  // tables return at once, without a draw.  `which` follows kDispNames.
  __device__ double fek(int which, double eet) {
    const DevTables &T = F.T;
    const bool emit = (which & 1) == 0;
    const int phon = which >> 1;  // 0 LO, 1 TO, 2 LA
    const double e = phon == 0 ? T.templog : (phon == 1 ? T.temptof : T.templaf);
    const double ie = eet / e;
    if (emit && ie < 1.0) return phon == 2 ? -1.0e-10 : 1.0e-10;
    // energy ranges: upper bound, offset, scale, first column, edeta
    double shift, mult, edeta;
    int base;
    bool last = false;
    if (phon == 0 && emit) {  // FEKLOEM
      if (ie < 3.05) { shift = 1.0; mult = 10.0; base = 0; edeta = 1.0; }
      else if (ie < 5.625) { shift = 3.0; mult = 4.0; base = 20; edeta = 2.0; }
      else if (ie < 13.25) { shift = 5.5; mult = 2.0; base = 30; edeta = 4.0; }
      else if (ie < 28.5) { shift = 13.0; mult = 1.0; base = 45; edeta = 8.0; }
      else { shift = 28.0; mult = 1.0; base = 60; edeta = 12.0; last = true; }
    } else if (phon == 0) {  // FEKLOAB
      if (ie < 1.05) { shift = 0.0; mult = 10.0; base = 0; edeta = 1.0; }
      else if (ie < 3.625) { shift = 1.0; mult = 4.0; base = 10; edeta = 2.0; }
      else if (ie < 11.25) { shift = 3.5; mult = 2.0; base = 20; edeta = 4.0; }
      else if (ie < 26.5) { shift = 11.0; mult = 1.0; base = 35; edeta = 8.0; }
      else { shift = 26.0; mult = 1.0; base = 50; edeta = 12.0; last = true; }
    } else if (emit) {  // FEKTOEM, FEKLAEM
      if (ie < 3.05) { shift = 1.0; mult = 10.0; base = 0; edeta = 0.25; }
      else if (ie < 5.625) { shift = 3.0; mult = 4.0; base = 20; edeta = 0.5; }
      else if (ie < 13.25) { shift = 5.5; mult = 2.0; base = 30; edeta = 0.5; }
      else { shift = 13.0; mult = 1.0; base = 45; edeta = 1.0; last = true; }
    } else {  // FEKTOAB, FEKLAAB
      if (ie < 1.05) { shift = 0.0; mult = 10.0; base = 0; edeta = 0.25; }
      else if (ie < 3.625) { shift = 1.0; mult = 4.0; base = 10; edeta = 0.25; }
      else if (ie < 11.25) { shift = 3.5; mult = 2.0; base = 20; edeta = 0.5; }
      else { shift = 11.0; mult = 1.0; base = 35; edeta = 1.0; last = true; }
    }
    int it = (int)((ie - shift) * mult + 0.5);
    if (it < 1) it = 1;
    if (last) {  // the last range's cap
      if (phon == 0) { if (it > 60) it = 60; }
      else if (emit) { if (it > 115) it = 115; }
      else if (it > 60) it = 115;  // as the reference: past 60 the column jumps to 150
    }
    const int ei = base + it;
    const int cols = phon == 0 ? (emit ? 120 : 110) : (emit ? 160 : 150);
    const int rows = phon == 0 ? 201 : 51;
    const double *tab = T.disp + T.disp_off[which] + (ei - 1);
    const double ran = (double)Random();
    int i = 0;
    double ksum = 0.0;
    if (which == 0) {  // FEKLOEM wraps before adding: rows 0..199
      while (ksum < ran) {
        ++i;
        if (i == rows) { ksum = 1.1; i = 1; }
        ksum += tab[(size_t)(i - 1) * cols];
      }
    } else {
      while (ksum < ran) {
        ++i;
        ksum += tab[(size_t)(i - 1) * cols];
        if (i == rows) { ksum = 1.1; i = 1; }
      }
    }
    const int j = i % 2, k = i / 2;
    const double c = phon == 0 ? 0.01 : 0.04;
    double ef;
    if (emit) ef = j == 1 ? eet - e * (1.0 - c * edeta * k) : eet - e * (1.0 + c * edeta * k);
    else ef = j == 1 ? eet + e * (1.0 + c * edeta * k) : eet + e * (1.0 - c * edeta * k);
    if (phon == 2 && ef <= 0.0) ef = 1.0e-5 * e;
    return ef;
  }

  // Set-up of EPSCAT (src/ElectronPhononScatter.cpp:98-195; with
  // Flag_QuantumCorrection the LO / LA / TO events take their final energy
  // from fek, :152-167), ESCATII (:406-497, seciifl = false), HPSCAT
  // (src/HolePhononScatter.cpp:86-146) and HSCATII (:149-234) for mechanism
  // iscat: the final band and energy, and the wedge rule of the draw
  // (fs_tal: 1..3 = TALIND(ityp), 0 = a random isym, -1 = none).
  __device__ void request_scatter(int iscat) {
    save_old();
    const DevTables &T = F.T;
    if (type == 0) {
      iband = iscat / T.scpre + T.bandof[0];
      const int m = iscat % T.scpre;
      if (m + 1 == T.scpre) {  // ESCATII
        fs_kind = kFsIonize;
        fs_tal = 0;
        energy = (energy - T.sieg) / 3.0;
        return;
      }
      fs_kind = kFsPhonon;
      switch (m) {
        case 0: fs_tal = 1; break;
        case 1: energy = energy + T.temptag; fs_tal = 2; break;
        case 2: energy = energy - T.temptag; fs_tal = 2; break;
        case 3: energy = energy + T.templag; fs_tal = 2; break;
        case 4: energy = energy - T.templag; fs_tal = 2; break;
        case 5: energy = energy + T.templog; fs_tal = 2; break;
        case 6: energy = energy - T.templog; fs_tal = 2; break;
        case 7: energy = energy + T.temptaf; fs_tal = 3; break;
        case 8: energy = energy - T.temptaf; fs_tal = 3; break;
        case 9: energy = energy + T.templaf; fs_tal = 3; break;
        case 10: energy = energy - T.templaf; fs_tal = 3; break;
        case 11: energy = energy + T.temptof; fs_tal = 3; break;
        case 12: energy = energy - T.temptof; fs_tal = 3; break;
        default: fs_tal = -1; break;
      }
      if (I->M.quantum && (m == 5 || m == 6 || (m >= 9 && m <= 12))) {
        // the dispersion table of the event: LO 5 / 6, LA 9 / 10, TO 11 / 12
        // (absorption / emission); the energy before the event
        static constexpr signed char kTable[13] = {-1, -1, -1, -1, -1, 1, 0, -1, -1, 5, 4, 3, 2};
        energy = fek(kTable[m], fs_eeold);
      }
    } else {
      iband = iscat / T.scprh + T.bandof[1];
      const int m = iscat % T.scprh;
      fs_tal = 0;
      if (m + 1 == T.scprh) {  // HSCATII
        fs_kind = kFsIonize;
        energy = (energy - T.sieg) / 3.0;
        return;
      }
      fs_kind = kFsPhonon;
      if (m == 1) energy = energy + T.temphop;
      else if (m == 2) energy = energy - T.temphop;
    }
  }
  // Set-up of Diffuse, src/CellHit.cpp:243-386 (TALIND(1), get_state, then
  // the mirror that points the velocity back into the device).
  __device__ void request_diffuse() {
    save_old();
    fs_kind = kFsDiffuse;
    fs_tal = 1;
  }
  // The draws and epilogue of the pending final state.
  __device__ void run_final_state() {
    const int kind = fs_kind;
    fs_kind = kFsNone;
    if (fs_tal == 0) isym = ((int)((R)48 * Random()) % 48);
    else if (fs_tal > 0) TALIND(fs_tal);
    get_state();
    if (kind == kFsDiffuse) {
      if (self) restore_k();
      GetV();
      switch (idir) {
        case kUp:
          if (vx == (R)0) restore_k();
          if (vx < (R)0) reflect_axis(0);
          break;
        case kRight:
          if (vy == (R)0) restore_k();
          if (vy > (R)0) reflect_axis(1);
          break;
        case kDown:
          if (vx == (R)0) restore_k();
          if (vx > (R)0) reflect_axis(0);
          break;
        case kLeft:
          if (vy == (R)0) restore_k();
          if (vy < (R)0) reflect_axis(1);
          break;
        case kFront:
          if (vz == (R)0) restore_k();
          if (vz < (R)0) reflect_axis(2);
          break;
        case kBack:
          if (vz == (R)0) restore_k();
          if (vz > (R)0) reflect_axis(2);
          break;
      }
      return;
    }
    if (self) {
      energy = fs_eeold;
      restore_k();
    }
    if (kind == kFsPhonon && I->M.heat)
      heat_to_point((energy - fs_eeold) * fabs(charge), type == 0 ? I->Y.heat_e : I->Y.heat_h);
  }

  // ElectronPhononScatter (src/ElectronPhononScatter.cpp:5-95) and
  // HolePhononScatter (src/HolePhononScatter.cpp:4-83): real or
  // self-scattering against the variable-gamma majorant; a real event
  // leaves the mechanism search to run_pick.
  __device__ void phonon_event() {
    const R scasum = CALSCATTSUM((R)energy, iband);
    const R g = tf(itet).gam;
    const R drand = scasum > g ? Random() * scasum : Random() * g;
    if (scasum < drand) {
      self = true;
      return;
    }
    self = false;
    pick_drand = drand;
    pick_pending = true;
  }
  // The mechanism search of ElectronPhononScatter / HolePhononScatter
  // (src/ElectronPhononScatter.cpp:47-63, src/HolePhononScatter.cpp:49-66).
  __device__ void run_pick() {
    pick_pending = false;
    const int iscat = type == 0 ? pick_electron_mechanism(pick_drand) : pick_hole_mechanism(pick_drand);
    if (iscat < 0) {
      self = true;
      return;
    }
    request_scatter(iscat);
  }

  // GetImpScRate, src/ElectronImpurityScatter.cpp:62-126 (Brooks-Herring,
  // bhmrtfl = false).  FP32: the same rate written as
  // imp_a * sqrt(e) / (1 + imp_b * e) with the cell's constants (load_cell_fields).
  __device__ R GetImpScRate(R eel) const {
    if constexpr (sizeof(R) == 4) {
      return eel < imp_ecut ? imp_a * m_sqrt(eel) / ((R)1 + imp_b * eel) : (R)0;
    } else {
      const DevTables &T = F.T;
      if ((eel * T.eV0 < 0.120) && (DA * T.conc0 >= 1e22)) {
        const double eebeta = T.frickel * 4 * kPiD * Rho / (2.0 * T.meld * T.eps_si);
        if (I->M.surface_scatter && I->M.surface_impurity && I->M.in_surf[cell_index()]) {
          // The reference's surface-impurity formula is commented out there and
          // leaves the rate unset; the engine treats it as zero.
          return 0.0;
        }
        const double fr = T.frickel * Rho;
        return DA * T.meld * sqrt(2.0 * T.meld * eel) /
               (kPiD * (fr * fr) * (1.0 + 4.0 * eel * T.melt / (eebeta * T.meld)));
      }
      return 0.0;
    }
  }

  // GetImpScGamma, src/ElectronImpurityScatter.cpp:6-59: majorant of the
  // BH rate over the tet's energy span.
  __device__ R GetImpScGamma() const {
    const DevTables &T = F.T;
    R eemax;
    if constexpr (sizeof(R) == 4) eemax = imp_emax;
    else eemax = T.frickel * 4 * kPiD * Rho / (8.0 * T.melt * T.eps_si);
    const TetFlightT<R> &s = tf(itet);
    R gammax;
    if (eemax < s.e0) gammax = GetImpScRate(s.e0);
    else if (eemax > s.e3) gammax = GetImpScRate(s.e3);
    else gammax = GetImpScRate(eemax);
    const R floor_ = (R)(1.0 / T.scrt0);
    return gammax > floor_ ? gammax : floor_;
  }

  // EleImpScUpdateK, src/ElectronImpurityScatter.cpp:188-306.
  __device__ void EleImpScUpdateK();

  // ElectronImpurityScatter, src/ElectronImpurityScatter.cpp:128-185.
  __device__ void ElectronImpurityScatter() {
    const R gamimp = GetImpScRate((R)energy);
    if (gamimp < Random() * imp_gamma) {
      self = true;
    } else {
      EleImpScUpdateK();
    }
  }

  // GetSurfScRate, src/ParSurfaceScatter.cpp:3-45.
  __device__ void GetSurfScRate() {
    const int c = cell_index();
    if (type == 0) { rough_rate = (R)I->M.e_rough[c]; sphon_rate = (R)I->M.e_sphon[c]; }
    else { rough_rate = (R)I->M.h_rough[c]; sphon_rate = (R)I->M.h_sphon[c]; }
    surf_gamma = rough_rate + sphon_rate;
  }

  __device__ void reflect_axis(int axis) {
    if (axis == 0) kx = -kx;
    else if (axis == 1) ky = -ky;
    else kz = -kz;
    isym = S.refl[axis * 48 + isym];
  }
  // Reflect, src/CellHit.cpp:214-240.
  __device__ void Reflect() {
    if (idir == kUp || idir == kDown) reflect_axis(0);
    else if (idir == kRight || idir == kLeft) reflect_axis(1);
    else if (idir == kFront || idir == kBack) reflect_axis(2);
  }
  __device__ bool inside_mesh(int i, int j, int k) const {
    return i >= 0 && j >= 0 && k >= 0 && i < I->M.nx && j < I->M.ny && k < I->M.nz;
  }
  // Pass, src/CellHit.cpp:389-413.  A PASS rule on the outer x / z boundary
  // would move the particle off the mesh (the reference indexes out of its
  // arrays there); the engine removes such a particle and counts it.
  __device__ void Pass() {
    int ni, nj, nk;
    neighbour(ni, nj, nk);
    if (!inside_mesh(ni, nj, nk)) {
      count(I->Y, kCntUnfinished);
      catch_ = true;
      return;
    }
    const DevMesh &M = I->M;
    if constexpr (Real::kCellRelative) {  // the face, in the new cell's frame
      switch (idir) {
        case kUp: x = M.dxf[ic - 1]; ic--; break;
        case kDown: x = 0; ic++; break;
        case kRight:
          y = 0;
          jc++;
          tally_add_i64(I->Y.rcurrent + jc, charge, kChargeScale);
          break;
        case kLeft:
          y = M.dyf[jc - 1];
          tally_add_i64(I->Y.lcurrent + jc, charge, kChargeScale);
          jc--;
          break;
        case kFront: z = M.dzf[kc - 1]; kc--; break;
        case kBack: z = 0; kc++; break;
      }
    } else {
      switch (idir) {
        case kUp: x = M.lx[ic]; ic--; break;
        case kDown: x = M.lx[ic + 1]; ic++; break;
        case kRight:
          y = M.ly[jc + 1];
          jc++;
          tally_add_i64(I->Y.rcurrent + jc, charge, kChargeScale);
          break;
        case kLeft:
          y = M.ly[jc];
          tally_add_i64(I->Y.lcurrent + jc, charge, kChargeScale);
          jc--;
          break;
        case kFront: z = M.lz[kc]; kc--; break;
        case kBack: z = M.lz[kc + 1]; kc++; break;
      }
    }
  }
  // Period, src/CellHit.cpp:416-432.
  __device__ void Period() {
    const DevMesh &M = I->M;
    if constexpr (Real::kCellRelative) {
      if (idir == kUp) x = M.dxf[ic];
      else if (idir == kDown) x = 0;
      else if (idir == kLeft) y = M.dyf[jc];
      else if (idir == kRight) y = 0;
      else if (idir == kFront) z = M.dzf[kc];
      else if (idir == kBack) z = 0;
    } else {
      if (idir == kUp) x = M.lx[ic + 1];
      else if (idir == kDown) x = M.lx[ic];
      else if (idir == kLeft) y = M.ly[jc + 1];
      else if (idir == kRight) y = M.ly[jc];
      else if (idir == kFront) z = M.lz[kc + 1];
      else if (idir == kBack) z = M.lz[kc];
    }
  }
  __device__ void neighbour(int &i, int &j, int &k) const {
    i = ic; j = jc; k = kc;
    switch (idir) {
      case kUp: i = ic - 1; break;
      case kDown: i = ic + 1; break;
      case kLeft: j = jc - 1; break;
      case kRight: j = jc + 1; break;
      case kFront: k = kc - 1; break;
      case kBack: k = kc + 1; break;
    }
  }
  __device__ void contact_add(int icont, int slot, double v, double scale) const {
    if (icont < 0 || icont >= kMaxContacts) return;
    tally_add_i64(I->Y.contact + icont * 6 + slot, v, scale);
  }
  // Generate, src/CellHit.cpp:435-501: tally, then a copy of the particle
  // enters the neighbour cell and finishes the step there.
  __device__ void Generate() {
    count(I->Y, kCntGenerated);
    const int icont = I->M.contact[cell_index()] - 1;
    if (icont >= 0) {
      atomicAdd(reinterpret_cast<unsigned long long *>(I->Y.contact + icont * 6 + 0), 1ull);
      contact_add(icont, 1, charge, kChargeScale);
      contact_add(icont, 2, energy, kEnergyScale);
    }
    if (idir == kRight) tally_add_i64(I->Y.rcurrent + jc + 1, charge, kChargeScale);
    if (idir == kLeft) tally_add_i64(I->Y.lcurrent + jc, charge, kChargeScale);
    int i, j, k;
    neighbour(i, j, k);
    if (!inside_mesh(i, j, k)) {
      count(I->Y, kCntUnfinished);
      return;
    }
    const DevChildrenT<R> &C = I->C;
    const unsigned slot = atomicAdd(C.count, 1u);
    const uint32_t csub = sub * 16u + 1u + (uint32_t)nchild++;
    if ((int)slot >= C.capacity) {
      count(I->Y, kCntChildOverflow);
      return;
    }
    R cx = x, cy = y, cz = z;
    if constexpr (Real::kCellRelative) {  // the same point in the neighbour cell's frame
      const DevMesh &M = I->M;
      switch (idir) {
        case kUp: cx = x + M.dxf[i]; break;
        case kDown: cx = x - M.dxf[ic]; break;
        case kLeft: cy = y + M.dyf[j]; break;
        case kRight: cy = y - M.dyf[jc]; break;
        case kFront: cz = z + M.dzf[k]; break;
        case kBack: cz = z - M.dzf[kc]; break;
      }
    }
    C.x[slot] = cx; C.y[slot] = cy; C.z[slot] = cz;
    C.kx[slot] = kx; C.ky[slot] = ky; C.kz[slot] = kz;
    C.energy[slot] = energy; C.charge[slot] = charge; C.left_time[slot] = left_time;
    C.cell[slot] = pack_cell(i, j, k);
    C.itet[slot] = itet;
    C.meta[slot] = (uint32_t)isym | ((uint32_t)type << 8);
    C.parent_uid[slot] = uid;
    C.sub[slot] = csub;
  }
  // CatchAtContact / CatchAtGate, src/CellHit.cpp:504-574.
  __device__ void Catch(bool with_current) {
    int i, j, k;
    neighbour(i, j, k);
    const int icont = inside_mesh(i, j, k) ? I->M.contact[cell_index(i, j, k)] - 1 : -1;
    if (with_current) {
      if (idir == kRight) tally_add_i64(I->Y.rcurrent + jc + 1, charge, kChargeScale);
      if (idir == kLeft) tally_add_i64(I->Y.lcurrent + jc, charge, kChargeScale);
    }
    if (icont >= 0 && icont < kMaxContacts) {
      atomicAdd(reinterpret_cast<unsigned long long *>(I->Y.contact + icont * 6 + 3), 1ull);
      contact_add(icont, 4, charge, kChargeScale);
      contact_add(icont, 2, energy, kEnergyScale);  // the reference adds to EnergyGen here (src/CellHit.cpp:542)
    }
  }
  __device__ void load_cell_fields() {
    const int c = cell_index();
    const DevMesh &M = I->M;
    if constexpr (sizeof(R) == 8) {
      const double *f = (type == 0 ? M.efield : M.hfield) + 3 * (size_t)c;
      Ex = f[0];
      Ey = f[1];
      Ez = f[2];
      Rho = M.rho[c];
      DA = M.da[c];
    } else {
      const float4 *r = M.cell32 + 3 * (size_t)c;
      if (type == 0) {
        const float4 a = r[0], b = r[1], m = r[2];
        Ex = a.x; Ey = a.y; Ez = a.z;
        imp_a = a.w;
        imp_b = b.w;
        imp_emax = m.x;
        imp_beta = m.y;
        imp_ecut = m.z;
      } else {
        const float4 b = r[1];
        Ex = b.x; Ey = b.y; Ez = b.z;
      }
    }
  }
  // HitCell, src/CellHit.cpp:96-211.  Returns false when the particle would
  // leave the device through a PASS / GENERATE face on the outer y boundary.
  __device__ bool HitCell() {
    const int imot = I->M.motion[(size_t)cell_index() * 6 + idir];
    if (imot == kPass || imot == kGenerate || imot == kGenRef) {
      if ((idir == kLeft && jc == 0) || (idir == kRight && jc == I->M.ny - 1)) return false;
    }
    if (imot == kPass) Pass();
    else if (imot == kReflect) Reflect();
    else if (imot == kScattOx) {
      if (I->M.surface_scatter) Reflect();
      else {
        if (Random() > (R)F.T.difpr[type]) Reflect();
        else request_diffuse();
      }
    } else if (imot == kPeriod) Period();
    else if (imot == kGenerate || imot == kGenRef) {
      Generate();
      Reflect();
    } else if (imot == kCatch) {
      Catch(true);
      catch_ = true;
    } else if (imot == kCatchGate) {
      Catch(false);
      catch_ = true;
    } else {
      catch_ = true;  // no such rule: the reference exits
      count(I->Y, kCntNoTet);
    }
    load_cell_fields();
    return true;
  }
  // ParticleSurfaceScatter, src/ParSurfaceScatter.cpp:48-61, with the
  // surface-phonon branches' drand defined (see file note).
  __device__ void surface_event() {
    if (Random() * surf_gamma < rough_rate) {
      idir = I->M.surface_dir[min(max(I->M.nearest_surf[cell_index()], 0), kMaxSurfaces - 1)];
      request_diffuse();
      return;
    }
    self = false;
    pick_drand = Random() * (type == 0 ? electron_rate_sum() : hole_rate_sum());
    pick_pending = true;
  }

  // One particle, one step: particle_fly, src/mcmodel.cpp:1874-2161, split
  // into begin (the set-up before the event loop), iterate (one pass of the
  // loop; true when the particle's step is over) and finish (the tallies
  // after the loop), so a kernel can interleave particles on one lane.
  // Loop state (particle_fly's locals):
  bool get_tet, get_cell, get_ph, get_imp, get_surf, too_far;
  R ssnl, imprnl, phrnl, TetTf, CellTf;
  int loop, zero_run;

  __device__ void begin() {
    catch_ = false;
    pick_pending = false;
    fs_kind = kFsNone;
    loc_mode = kLocNone;
    get_tet = get_cell = get_ph = get_imp = get_surf = true;
    ssnl = imprnl = phrnl = 0;
    TetTf = CellTf = 0;
    too_far = false;
    zero_run = 0;
    load_cell_fields();
    iband = tf(itet).band;
    GetV();
    loop = 0;
    surf_gamma = 0;
    imp_gamma = 0;
  }

  __device__ bool iterate() {
    GetV();
    if (++loop > kMaxEvents) {
      count(I->Y, kCntTooManyEvents);
      catch_ = true;
      return true;
    }
    if (get_tet) { TetTf = TetTime(); get_tet = false; }
    if (get_cell) { CellTf = CellTime(); get_cell = false; }
    if (get_ph) { phrnl = -m_log(Random()); get_ph = false; }
    const R g = tf(itet).gam;
    R PhScTf, ImpScTf, SurfScTf, Tf;
    PhScTf = phrnl / g;
    if (iband == F.T.bandof[0]) {
      if (get_imp) { imprnl = -m_log(Random()); get_imp = false; }
      imp_gamma = GetImpScGamma();
      ImpScTf = imprnl / imp_gamma;
    } else {
      ImpScTf = (R)(2 * I->dt);
      imp_gamma = (R)(1.0 / F.T.scrt0);
    }
    if (I->M.surface_scatter && I->M.in_surf[cell_index()]) {
      if (get_surf) { ssnl = -m_log(Random()); get_surf = false; }
      GetSurfScRate();
      SurfScTf = (surf_gamma > 0 && ssnl > 0) ? ssnl / surf_gamma : (R)(2 * I->dt);
    } else {
      SurfScTf = (R)(2 * I->dt);
    }
    // Min(..., flag), src/Constant_GlobalVariable_MathFunction.cpp:92-118
    int flag = 1;
    Tf = TetTf;
    if (Tf > CellTf) { Tf = CellTf; flag = 2; }
    if (Tf > PhScTf) { Tf = PhScTf; flag = 3; }
    if (Tf > ImpScTf) { Tf = ImpScTf; flag = 4; }
    if (Tf > SurfScTf) { Tf = SurfScTf; flag = 5; }
    if ((double)Tf > left_time) { Tf = (R)left_time; flag = 6; }
    if constexpr (sizeof(R) == 8) {
      if (Tf < kMyZero) {
        catch_ = true;
        return true;
      }
    } else {
      // float event times that round to zero (or below) are events now
      if (!(Tf > (R)0)) {
        Tf = 0;
        if (++zero_run > kMaxZeroTimeEvents) {
          count(I->Y, kCntZeroTime);
          catch_ = true;
          return true;
        }
      } else {
        zero_run = 0;
      }
    }
    TetTf -= Tf;
    CellTf -= Tf;
    PhScTf -= Tf;
    ImpScTf -= Tf;
    SurfScTf -= Tf;
    if constexpr (MCB200_FLIGHT_EVENT_STATS != 0)
      count(I->Y, flag == 1 ? kStatTetFace : flag == 2 ? kStatCellFace : flag == 6 ? kStatStepEnd : kStatScatter);
    if (flag == 6) left_time = 0;  // Tf == left_time: the step is used up
    else left_time -= Tf;
    phrnl -= g * Tf;
    imprnl -= imp_gamma * Tf;
    ssnl -= surf_gamma * Tf;
    kx += Ex * Tf;
    ky += Ey * Tf;
    kz += Ez * Tf;
    energy += (vx * Ex + vy * Ey + vz * Ez) * Tf;
    x += vx * Tf;
    y += vy * Tf;
    z += vz * Tf;
    if (energy < 0) {
      catch_ = true;
      return true;
    }
    switch (flag) {
      case 1:
        HitTet();
        get_tet = true;
        get_cell = true;
        break;
      case 2:
        if (HitCell()) {
          get_tet = true;
          get_cell = true;
        } else {
          // trace_back, src/mcmodel.cpp:1774-1783
          kx -= Ex * Tf;
          ky -= Ey * Tf;
          kz -= Ez * Tf;
          energy -= (vx * Ex + vy * Ey + vz * Ez) * Tf;
          x -= vx * Tf;
          y -= vy * Tf;
          z -= vz * Tf;
          left_time += Tf;
          too_far = true;
        }
        break;
      case 3:
        phonon_event();
        break;
      case 4:
        if (type == 0) ElectronImpurityScatter();
        break;
      case 5:
        surface_event();
        break;
    }
    // shared tails: mechanism search, final-state draw, k-point search
    if (pick_pending) run_pick();
    if (fs_kind != kFsNone) run_final_state();
    if (loc_mode != kLocNone) run_locate();
    if (flag == 3) {
      if (!self) {
        get_tet = true;
        get_cell = true;
        count(I->Y, kCntPhonon);
      }
      get_ph = true;
    } else if (flag == 4) {
      if (!self) {
        get_tet = true;
        get_cell = true;
        count(I->Y, kCntImpurity);
      }
      get_imp = true;
    } else if (flag == 5) {
      if (!self) {
        get_tet = true;
        get_cell = true;
      }
      get_surf = true;
    }
    if (too_far || catch_) return true;
    return !(left_time > 0);
  }

  // Returns 0 done, 1 caught, 2 unfinished (outer-boundary PASS).  A
  // caller that sums the particles' event counts itself (`loop`, one
  // simulation per launch) passes kCountEvents = false.
  template <bool kCountEvents = true>
  __device__ int finish() {
    if constexpr (kCountEvents) atomicAdd(&I->Y.counters[kCntEvents], (unsigned long long)loop);
    if (catch_) {
      count(I->Y, kCntCaught);
      return 1;
    }
    if (too_far) {
      count(I->Y, kCntUnfinished);
      return 2;
    }
    return 0;
  }

  __device__ int fly() {
    begin();
    if (left_time > 0)
      while (!iterate()) {
      }
    return finish();
  }
};
using Flyer = FlyerT<double>;

}  // namespace mcb200
