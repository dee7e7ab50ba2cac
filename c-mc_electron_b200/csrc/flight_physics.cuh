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

// Symmetry tables staged in shared memory (one copy per block).
struct SymSmem {
  int symi[48 * 6];   // matsym[c][s] at s*6+c
  int newisym[5 * 48];
  double bz[3 * 5 * 48];
  int refl[3 * 48];
};

struct FlightCtx {
  DevTables T;
  DevMesh M;
  DevTallies Y;
  DevChildren C;
  double dt;
  uint64_t seed;
  uint32_t step;
};

__device__ __forceinline__ void tally_add_i64(long long *p, double v, double scale) {
  atomicAdd(reinterpret_cast<unsigned long long *>(p), (unsigned long long)__double2ll_rn(v * scale));
}
__device__ __forceinline__ void count(const DevTallies &Y, int which) { atomicAdd(&Y.counters[which], 1ull); }

struct Flyer {
  const FlightCtx &F;
  const SymSmem &S;
  // random stream
  uint32_t uid, sub, n;
  // particle registers (MeshQuantities members, include/mcmodel.h:215-233)
  double x, y, z, kx, ky, kz, energy, charge, left_time;
  int ic, jc, kc, itet, isym, type, iband;
  double Ex, Ey, Ez, Rho, DA, vx, vy, vz;
  int itetdir, idir;
  bool catch_, self;
  double rough_rate, sphon_rate, surf_gamma, imp_gamma;
  int nchild;

  __device__ Flyer(const FlightCtx &f, const SymSmem &s) : F(f), S(s) {}

  __device__ __forceinline__ double Random() { return mcb200_uniform(F.seed, uid, F.step, sub, n++); }

  __device__ __forceinline__ int ms(int c, int s) const { return S.symi[s * 6 + c]; }
  __device__ __forceinline__ int cell_index() const { return (jc * F.M.nx + ic) * F.M.nz + kc; }
  __device__ __forceinline__ int cell_index(int i, int j, int k) const { return (j * F.M.nx + i) * F.M.nz + k; }

  // in_wedge, src/ParticleUtils.cpp:295-305: BZ vector -> irreducible wedge of isym.
  __device__ __forceinline__ void in_wedge(double &xo, double &yo, double &zo, double xi, double yi, double zi) const {
    const int p0 = ms(0, isym) - 1, p1 = ms(1, isym) - 1;
    const double a = xi * (double)ms(3, isym), b = yi * (double)ms(4, isym), c = zi * (double)ms(5, isym);
    xo = p0 == 0 ? a : (p1 == 0 ? b : c);
    yo = p0 == 1 ? a : (p1 == 1 ? b : c);
    zo = p0 == 2 ? a : (p1 == 2 ? b : c);
  }
  // Band::OutWedge, src/Band.cpp:555-570: wedge vector -> BZ.
  __device__ __forceinline__ void out_wedge(double &xo, double &yo, double &zo, double xi, double yi, double zi) const {
    const int p0 = ms(0, isym) - 1, p1 = ms(1, isym) - 1, p2 = ms(2, isym) - 1;
    xo = (p0 == 0 ? xi : (p0 == 1 ? yi : zi)) * (double)ms(3, isym);
    yo = (p1 == 0 ? xi : (p1 == 1 ? yi : zi)) * (double)ms(4, isym);
    zo = (p2 == 0 ? xi : (p2 == 1 ? yi : zi)) * (double)ms(5, isym);
  }
  // GetV, src/ParticleUtils.cpp:307-313.
  __device__ __forceinline__ void GetV() {
    const double4 v = *reinterpret_cast<const double4 *>(F.T.tf[itet].v);
    out_wedge(vx, vy, vz, v.x, v.y, v.z);
  }
  // GetEnergy, src/ParticleUtils.cpp:315-329.
  __device__ void GetEnergy() {
    double dx, dy, dz;
    in_wedge(dx, dy, dz, kx, ky, kz);
    const double4 k0 = F.T.knode[F.T.tnode[itet].x];
    dx -= k0.x;
    dy -= k0.y;
    dz -= k0.z;
    const double *v = F.T.tf[itet].v;
    energy = v[3] + v[0] * dx + v[1] * dy + v[2] * dz;
  }
  __device__ __forceinline__ double face_dist(int it, int f, double a, double b, double c) const {
    const double *nn = F.T.tf[it].n[f];
    return nn[0] * a + nn[1] * b + nn[2] * c - nn[3];
  }
  __device__ __forceinline__ bool tet_contains(int it, double a, double b, double c) const {
    return face_dist(it, 0, a, b, c) >= -kMyZero && face_dist(it, 1, a, b, c) >= -kMyZero &&
           face_dist(it, 2, a, b, c) >= -kMyZero && face_dist(it, 3, a, b, c) >= -kMyZero;
  }

  // TetTime, src/TetHit.cpp:4-106: time to the tet face the drift reaches first.
  __device__ double TetTime() {
    double xkl, ykl, zkl, xfl, yfl, zfl;
    in_wedge(xkl, ykl, zkl, kx, ky, kz);
    in_wedge(xfl, yfl, zfl, Ex, Ey, Ez);
    const TetFlight &t = F.T.tf[itet];
    double best = 0;
    itetdir = 0;
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      const double nf = t.n[f][0] * xfl + t.n[f][1] * yfl + t.n[f][2] * zfl;
      double tfp;
      if (nf < 0) {
        tfp = (t.n[f][3] - (t.n[f][0] * xkl + t.n[f][1] * ykl + t.n[f][2] * zkl)) / nf;
        if (tfp < 0) tfp = 0;
      } else {
        tfp = 1e99;
      }
      if (f == 0) best = tfp;
      else if (tfp < best) {
        best = tfp;
        itetdir = f;
      }
    }
    return best;
  }

  // CellTime, src/CellHit.cpp:4-93: time to the real-space cell face.
  __device__ double CellTime() {
    const DevMesh &M = F.M;
    int idx, idy, idz;
    double tx, ty, tz;
    if (vx > 0) { idx = kDown; tx = (M.lx[ic + 1] - x) / vx; }
    else if (vx < 0) { idx = kUp; tx = -(x - M.lx[ic]) / vx; }
    else { idx = kUp; tx = 1e99; }
    if (vy > 0) { idy = kRight; ty = (M.ly[jc + 1] - y) / vy; }
    else if (vy < 0) { idy = kLeft; ty = -(y - M.ly[jc]) / vy; }
    else { idy = kRight; ty = 1e99; }
    if (vz > 0) { idz = kBack; tz = (M.lz[kc + 1] - z) / vz; }
    else if (vz < 0) { idz = kFront; tz = -(z - M.lz[kc]) / vz; }
    else { idz = kFront; tz = 1e99; }
    idir = idx;
    double t = tx;
    if (ty < t) { idir = idy; t = ty; }
    if (tz < t) { idir = idz; t = tz; }
    if (t < -kMyZero) t = 0;
    return t;
  }

  // Band::CONFBZ, src/Band.cpp:573-616: fold k back into the first BZ.
  __device__ void CONFBZ(double &a, double &b, double &c) const {
    const double p = F.T.a0pi;
    for (int guard = 0; guard < 64; ++guard) {
      bool out = fabs(a) > p || fabs(b) > p || fabs(c) > p || fabs(a) + fabs(b) + fabs(c) > 1.50 * p;
      if (!out) return;
      a = a > 0.0 ? a - p : a + p;
      b = b > 0.0 ? b - p : b + p;
      c = c > 0.0 ? c - p : c + p;
    }
  }

  // Point location by walking the tetrahedral mesh: from `start`, repeatedly
  // step through the face whose plane the point lies furthest outside of,
  // until every face test passes (the reference's containment test,
  // d >= -MY_ZERO).  Returns -1 when the walk reaches a wedge boundary or
  // does not settle within the step cap; the caller then uses the k-grid.
  __device__ int walk_to(int start, double a, double b, double c) const {
    int it = start;
    for (int s = 0; s < 64; ++s) {
      int fmin = -1;
      double dmin = -kMyZero;
#pragma unroll
      for (int f = 0; f < 4; ++f) {
        const double d = face_dist(it, f, a, b, c);
        if (d < dmin) {
          dmin = d;
          fmin = f;
        }
      }
      if (fmin < 0) return it;
      const int nb = (&F.T.tneib[it].x)[fmin];
      if (nb < 0) return -1;
      it = nb;
    }
    return -1;
  }

  // Getisym, src/ParticleUtils.cpp:395-625: wedge from k, then the tet of
  // band iband that contains the wedge vector (k-grid lookup, see file note).
  __device__ void Getisym() {
    int mink, maxk;
    double tmin, tmax;
    if (fabs(kx) > fabs(ky)) { tmin = fabs(ky); tmax = fabs(kx); mink = 1; maxk = 0; }
    else { tmin = fabs(kx); tmax = fabs(ky); mink = 0; maxk = 1; }
    if (fabs(kz) < tmin) mink = 2;
    else if (fabs(kz) > tmax) maxk = 2;
    // pos[mink] = 2, pos[maxk] = 0, else 1 (mink != maxk always)
    const int p0 = maxk == 0 ? 0 : (mink == 0 ? 2 : 1);
    const int p1 = maxk == 1 ? 0 : (mink == 1 ? 2 : 1);
    const int p2 = maxk == 2 ? 0 : (mink == 2 ? 2 : 1);
    auto sgn = [](double v) { return (int)(fabs(v) / v); };  // utils.cpp sign()
    const int sx = sgn(kx) + 1, sy = sgn(ky) + 1, sz = sgn(kz) + 1;
    if (sx < 0 || sx > 2 || sy < 0 || sy > 2 || sz < 0 || sz > 2) {  // a zero component: sign() is NaN in the reference
      count(F.Y, kCntNoTet);
      catch_ = true;
      return;
    }
    isym = F.T.indmat[((((sx * 3 + sy) * 3 + sz) * 3 + p0) * 3 + p1) * 3 + p2];
    double a, b, c;
    in_wedge(a, b, c, kx, ky, kz);
    if (iband == F.T.ibt[itet] && tet_contains(itet, a, b, c)) return;
    int start = iband == F.T.ibt[itet] ? itet : -1;
    if (iband == F.T.bandof[0]) {  // lowest conduction band: start next to the point
      const int sg = kSeedGridN;
      const int si = min(max((int)floor((a - F.T.grid_lo[0]) * F.T.seed_inv[0]), 0), sg - 1);
      const int sj = min(max((int)floor((b - F.T.grid_lo[1]) * F.T.seed_inv[1]), 0), sg - 1);
      const int sk = min(max((int)floor((c - F.T.grid_lo[2]) * F.T.seed_inv[2]), 0), sg - 1);
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
    int gi = (int)floor((a - F.T.grid_lo[0]) * F.T.grid_inv[0]);
    int gj = (int)floor((b - F.T.grid_lo[1]) * F.T.grid_inv[1]);
    int gk = (int)floor((c - F.T.grid_lo[2]) * F.T.grid_inv[2]);
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
    count(F.Y, kCntNoTet);
    catch_ = true;
  }

  // GetisymBZ, src/ParticleUtils.cpp:331-392: after a BZ-boundary crossing,
  // search the BZ-surface tets of the particle's energy bin.
  __device__ void GetisymBZ() {
    double a, b, c;
    in_wedge(a, b, c, kx, ky, kz);
    if (iband == F.T.ibt[itet] && tet_contains(itet, a, b, c)) return;
    int ie = (int)(energy * F.T.dlist);
    if (ie < 0) ie = 0;
    if (ie >= kMWLE) ie = kMWLE - 1;
    const int p = F.T.pslist[ie * kMNB + iband], cnt = F.T.nslist[ie * kMNB + iband];
    for (int itl = p; itl <= p + cnt - 1; ++itl) {
      const int it = F.T.slist[itl];
      if (iband == F.T.ibt[it] && tet_contains(it, a, b, c)) {
        itet = it;
        return;
      }
    }
    Getisym();
  }

  // HitTet, src/TetHit.cpp:109-142.
  __device__ void HitTet() {
    const int nb = (&F.T.tneib[itet].x)[itetdir];
    if (nb >= 0) {
      itet = nb;
    } else if (nb == -5 || nb == -6) {
      const int ii = -nb - 2;
      kx = kx + S.bz[(0 * 5 + ii) * 48 + isym];
      ky = ky + S.bz[(1 * 5 + ii) * 48 + isym];
      kz = kz + S.bz[(2 * 5 + ii) * 48 + isym];
      isym = S.newisym[ii * 48 + isym];
      GetisymBZ();
      if (catch_) return;
      GetEnergy();
    } else {
      isym = S.newisym[(-nb - 2) * 48 + isym];
    }
  }

  // TALIND, src/ParticleUtils.cpp:626-748: final valley (and a random wedge
  // in it).  The reference's talend[] lookups are written as arithmetic on
  // the drawn index (1..4); an index of 5 (u*4+1 rounding up to 5, possible
  // only for u within 2^-51 of 1) reads past the reference's table and is
  // clamped to 4 here.
  __device__ __forceinline__ int talend_index() { return min((int)(Random() * 4.0 + 1.0), 4); }
  __device__ void TALIND(int ityp) {
    int ital = 1;
    const double ax = fabs(kx), ay = fabs(ky), az = fabs(kz);
    if (ax >= ay && ax >= az) {
      if (kx >= 0.0) {
        if (ityp == 1) ital = 1;
        if (ityp == 2) ital = 2;
        if (ityp == 3) ital = talend_index() + 2;  // {3,4,5,6}
      }
      if (kx < 0.0) {
        if (ityp == 1) ital = 2;
        if (ityp == 2) ital = 1;
        if (ityp == 3) ital = talend_index() + 2;
      }
    }
    if (ay >= az && ay >= ax) {
      if (ky >= 0.0) {
        if (ityp == 1) ital = 3;
        if (ityp == 2) ital = 4;
        if (ityp == 3) { const int i = talend_index(); ital = i <= 2 ? i : i + 2; }  // {1,2,5,6}
      }
      if (ky < 0.0) {
        if (ityp == 1) ital = 4;
        if (ityp == 2) ital = 3;
        if (ityp == 3) { const int i = talend_index(); ital = i <= 2 ? i : i + 2; }
      }
    }
    if (az > ay && az > ax) {
      if (kz >= 0.0) {
        if (ityp == 1) ital = 5;
        if (ityp == 2) ital = 6;
        if (ityp == 3) ital = talend_index();  // {1,2,3,4}
      }
      if (kz < 0.0) {
        if (ityp == 1) ital = 6;
        if (ityp == 2) ital = 5;
        if (ityp == 3) ital = talend_index();
      }
    }
    isym = (int)(Random() * 8.0) + 8 * (ital - 1);
  }

  // Band::CALDOSTETMAX, src/Band.cpp:2298-2320.
  __device__ double CALDOSTETMAX(double eed, int ib) const {
    const double *d = F.T.dostetmax + (size_t)ib * kNT;
    if (eed <= 0.0) return d[0];
    if (eed >= F.T.emax) return d[kNT - 1];
    const int itab = min((int)(eed / F.T.dtable), kNT - 2);  // eed just below emax may round to the last point
    return d[itab] > d[itab + 1] ? d[itab] : d[itab + 1];
  }

  // Band::SURF, src/Band.cpp:194-332 (only reached by FASTSURF for
  // tetrahedra whose two lowest nodes are degenerate).
  __device__ double SURF(double eps, int it) const;
  // Band::FASTSURF, src/Band.cpp:665-704.
  __device__ double FASTSURF(double eps, int it) const {
    const TetShape &s = F.T.ts[it];
    const double e0 = s.e[0], e1 = s.e[1], e2 = s.e[2], e3 = s.e[3];
    if (eps > e0 && eps < e3) {
      if (eps <= e1) return s.fac[0] * (eps - e0) * (eps - e0);
      if (eps < e2) {
        if (e1 - e0 > 1e-10) return s.fac[0] * (eps - e0) * (eps - e0) - s.fac[1] * (eps - e1) * (eps - e1);
        return SURF(eps, it);
      }
      return s.fac[2] * (eps - e3) * (eps - e3);
    }
    return 0.0;
  }

  // get_state, src/ParticleUtils.cpp:48-120: random final state on the
  // iso-energy surface of band iband (rejection on the tet's DOS share).
  __device__ void get_state() {
    if (energy <= 0.0) {
      self = true;
      return;
    }
    const double maxdostet = CALDOSTETMAX(energy, iband);
    int itab = (int)(energy * F.T.dlists);
    bool small_ = itab < kMWLES;
    if (!small_) {
      itab = (int)(energy * F.T.dlist);
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
      itet = lst[(int)(nted * Random()) + base];
      count2++;
      const TetShape &s = F.T.ts[itet];
      if ((count2 < 10000) && !((s.e[0] < energy) && (s.e[3] > energy))) continue;
      const double dostet = FASTSURF(energy, itet) / s.vgt;
      if (((Random() * maxdostet) > dostet) && (count2 < 10000)) continue;
      break;
    }
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
  __device__ double CALSCATTSUM(double eed, int ib) const {
    const double *s = F.T.sumscatt;
    if (eed <= 0.0) return s[ib];
    if (eed >= F.T.emax) return s[(size_t)(kNT - 1) * kMNB + ib];
    const int itab = min((int)(eed / F.T.dtable), kNT - 2);
    const double intp = (eed - F.T.energy[itab]) / (F.T.energy[itab + 1] - F.T.energy[itab]);
    return s[(size_t)itab * kMNB + ib] + intp * (s[(size_t)(itab + 1) * kMNB + ib] - s[(size_t)itab * kMNB + ib]);
  }

  // Electron mechanism choice by a running sum over Band::CALSCATTE
  // (src/Band.cpp:2165-2231) entries, without materialising the 56-entry
  // array: returns the chosen index or -1 (self-scattering).
  __device__ int pick_electron_mechanism(double drand) const;
  __device__ double electron_rate_sum() const;
  __device__ int pick_hole_mechanism(double drand) const;
  __device__ double hole_rate_sum() const;

  // heat_to_point, src/heat.cpp:169-196 (CIC onto the cell's 8 nodes).
  __device__ void heat_to_point(double e, long long *heat) const {
    const DevMesh &M = F.M;
    const double rx = (x - M.lx[ic]) / M.dx[ic];
    const double ry = (y - M.ly[jc]) / M.dy[jc];
    const double rz = (z - M.lz[kc]) / M.dz[kc];
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

  // EPSCAT, src/ElectronPhononScatter.cpp:98-195 (Flag_QuantumCorrection = 0).
  __device__ void EPSCAT(int iscat) {
    const double eeold = energy, xkold = kx, ykold = ky, zkold = kz;
    const int ibold = iband, itetold = itet, isymold = isym;
    const DevTables &T = F.T;
    iband = iscat / T.scpre + T.bandof[0];
    switch (iscat % T.scpre) {
      case 0: TALIND(1); break;
      case 1: energy = energy + T.temptag; TALIND(2); break;
      case 2: energy = energy - T.temptag; TALIND(2); break;
      case 3: energy = energy + T.templag; TALIND(2); break;
      case 4: energy = energy - T.templag; TALIND(2); break;
      case 5: energy = energy + T.templog; TALIND(2); break;
      case 6: energy = energy - T.templog; TALIND(2); break;
      case 7: energy = energy + T.temptaf; TALIND(3); break;
      case 8: energy = energy - T.temptaf; TALIND(3); break;
      case 9: energy = energy + T.templaf; TALIND(3); break;
      case 10: energy = energy - T.templaf; TALIND(3); break;
      case 11: energy = energy + T.temptof; TALIND(3); break;
      case 12: energy = energy - T.temptof; TALIND(3); break;
      default: break;
    }
    get_state();
    if (self) {
      energy = eeold; kx = xkold; ky = ykold; kz = zkold;
      iband = ibold; itet = itetold; isym = isymold;
    }
    if (F.M.heat) heat_to_point((energy - eeold) * fabs(charge), F.Y.heat_e);
  }

  // ESCATII, src/ElectronPhononScatter.cpp:406-497 (secondary generation off: seciifl = false).
  __device__ void ESCATII(int iscat) {
    const double eeold = energy, xkold = kx, ykold = ky, zkold = kz;
    const int ibold = iband, itetold = itet, isymold = isym;
    iband = iscat / F.T.scpre + F.T.bandof[0];
    energy = (energy - F.T.sieg) / 3.0;
    isym = ((int)(48 * Random()) % 48);
    get_state();
    if (self) {
      energy = eeold; kx = xkold; ky = ykold; kz = zkold;
      iband = ibold; itet = itetold; isym = isymold;
    }
  }

  // ElectronPhononScatter, src/ElectronPhononScatter.cpp:5-95.
  __device__ void ElectronPhononScatter() {
    const double scasum = CALSCATTSUM(energy, iband);
    const double g = F.T.gamtet[itet];
    const double drand = scasum > g ? Random() * scasum : Random() * g;
    if (scasum < drand) {
      self = true;
      return;
    }
    self = false;
    const int iscat = pick_electron_mechanism(drand);
    if (iscat < 0) {
      self = true;
      return;
    }
    if (((iscat % F.T.scpre) + 1) == F.T.scpre) ESCATII(iscat);
    else EPSCAT(iscat);
  }

  // HPSCAT, src/HolePhononScatter.cpp:86-146.
  __device__ void HPSCAT(int iscat) {
    const double eeold = energy, xkold = kx, ykold = ky, zkold = kz;
    const int ibold = iband, itetold = itet, isymold = isym;
    iband = iscat / F.T.scprh + F.T.bandof[1];
    switch (iscat % F.T.scprh) {
      case 1: energy = energy + F.T.temphop; break;
      case 2: energy = energy - F.T.temphop; break;
      default: break;
    }
    isym = ((int)(48 * Random()) % 48);
    get_state();
    if (self) {
      energy = eeold; kx = xkold; ky = ykold; kz = zkold;
      iband = ibold; itet = itetold; isym = isymold;
    }
    if (F.M.heat) heat_to_point((energy - eeold) * fabs(charge), F.Y.heat_h);
  }

  // HSCATII, src/HolePhononScatter.cpp:149-234 (seciifl = false).
  __device__ void HSCATII(int iscat) {
    const double eeold = energy, xkold = kx, ykold = ky, zkold = kz;
    const int ibold = iband, itetold = itet, isymold = isym;
    iband = iscat / F.T.scprh + F.T.bandof[1];
    energy = (energy - F.T.sieg) / 3.0;
    isym = ((int)(48 * Random()) % 48);
    get_state();
    if (self) {
      energy = eeold; kx = xkold; ky = ykold; kz = zkold;
      iband = ibold; itet = itetold; isym = isymold;
    }
  }

  // HolePhononScatter, src/HolePhononScatter.cpp:4-83.
  __device__ void HolePhononScatter() {
    const double scasum = CALSCATTSUM(energy, iband);
    const double g = F.T.gamtet[itet];
    const double drand = scasum > g ? Random() * scasum : Random() * g;
    if (scasum < drand) {
      self = true;
      return;
    }
    self = false;
    const int iscat = pick_hole_mechanism(drand);
    if (iscat < 0) {
      self = true;
      return;
    }
    if (((iscat % F.T.scprh) + 1) == F.T.scprh) HSCATII(iscat);
    else HPSCAT(iscat);
  }

  // GetImpScRate, src/ElectronImpurityScatter.cpp:62-126 (Brooks-Herring, bhmrtfl = false).
  __device__ double GetImpScRate(double eel) const {
    const DevTables &T = F.T;
    if ((eel * T.eV0 < 0.120) && (DA * T.conc0 >= 1e22)) {
      const double eebeta = T.frickel * 4 * kPiD * Rho / (2.0 * T.meld * T.eps_si);
      if (F.M.surface_scatter && F.M.surface_impurity && F.M.in_surf[cell_index()]) {
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

  // GetImpScGamma, src/ElectronImpurityScatter.cpp:6-59: majorant of the
  // BH rate over the tet's energy span.
  __device__ double GetImpScGamma() const {
    const DevTables &T = F.T;
    const double eemax = T.frickel * 4 * kPiD * Rho / (8.0 * T.melt * T.eps_si);
    const TetShape &s = T.ts[itet];
    double gammax;
    if (eemax < s.e[0]) gammax = GetImpScRate(s.e[0]);
    else if (eemax > s.e[3]) gammax = GetImpScRate(s.e[3]);
    else gammax = GetImpScRate(eemax);
    const double floor_ = 1.0 / T.scrt0;
    return gammax > floor_ ? gammax : floor_;
  }

  // EleImpScUpdateK, src/ElectronImpurityScatter.cpp:188-306.
  __device__ void EleImpScUpdateK();

  // ElectronImpurityScatter, src/ElectronImpurityScatter.cpp:128-185.
  __device__ void ElectronImpurityScatter() {
    const double gamimp = GetImpScRate(energy);
    if (gamimp < Random() * imp_gamma) {
      self = true;
    } else {
      EleImpScUpdateK();
    }
  }

  // GetSurfScRate, src/ParSurfaceScatter.cpp:3-45.
  __device__ void GetSurfScRate() {
    const int c = cell_index();
    if (type == 0) { rough_rate = F.M.e_rough[c]; sphon_rate = F.M.e_sphon[c]; }
    else { rough_rate = F.M.h_rough[c]; sphon_rate = F.M.h_sphon[c]; }
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
  // Diffuse, src/CellHit.cpp:243-386.
  __device__ void Diffuse();
  __device__ bool inside_mesh(int i, int j, int k) const {
    return i >= 0 && j >= 0 && k >= 0 && i < F.M.nx && j < F.M.ny && k < F.M.nz;
  }
  // Pass, src/CellHit.cpp:389-413.  A PASS rule on the outer x / z boundary
  // would move the particle off the mesh (the reference indexes out of its
  // arrays there); the engine removes such a particle and counts it.
  __device__ void Pass() {
    int ni, nj, nk;
    neighbour(ni, nj, nk);
    if (!inside_mesh(ni, nj, nk)) {
      count(F.Y, kCntUnfinished);
      catch_ = true;
      return;
    }
    const DevMesh &M = F.M;
    switch (idir) {
      case kUp: x = M.lx[ic]; ic--; break;
      case kDown: x = M.lx[ic + 1]; ic++; break;
      case kRight:
        y = M.ly[jc + 1];
        jc++;
        tally_add_i64(F.Y.rcurrent + jc, charge, kChargeScale);
        break;
      case kLeft:
        y = M.ly[jc];
        tally_add_i64(F.Y.lcurrent + jc, charge, kChargeScale);
        jc--;
        break;
      case kFront: z = M.lz[kc]; kc--; break;
      case kBack: z = M.lz[kc + 1]; kc++; break;
    }
  }
  // Period, src/CellHit.cpp:416-432.
  __device__ void Period() {
    const DevMesh &M = F.M;
    if (idir == kUp) x = M.lx[ic + 1];
    else if (idir == kDown) x = M.lx[ic];
    else if (idir == kLeft) y = M.ly[jc + 1];
    else if (idir == kRight) y = M.ly[jc];
    else if (idir == kFront) z = M.lz[kc + 1];
    else if (idir == kBack) z = M.lz[kc];
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
    tally_add_i64(F.Y.contact + icont * 6 + slot, v, scale);
  }
  // Generate, src/CellHit.cpp:435-501: tally, then a copy of the particle
  // enters the neighbour cell and finishes the step there.
  __device__ void Generate() {
    count(F.Y, kCntGenerated);
    const int icont = F.M.contact[cell_index()] - 1;
    if (icont >= 0) {
      atomicAdd(reinterpret_cast<unsigned long long *>(F.Y.contact + icont * 6 + 0), 1ull);
      contact_add(icont, 1, charge, kChargeScale);
      contact_add(icont, 2, energy, kEnergyScale);
    }
    if (idir == kRight) tally_add_i64(F.Y.rcurrent + jc + 1, charge, kChargeScale);
    if (idir == kLeft) tally_add_i64(F.Y.lcurrent + jc, charge, kChargeScale);
    int i, j, k;
    neighbour(i, j, k);
    if (!inside_mesh(i, j, k)) {
      count(F.Y, kCntUnfinished);
      return;
    }
    const DevChildren &C = F.C;
    const unsigned slot = atomicAdd(C.count, 1u);
    const uint32_t csub = sub * 16u + 1u + (uint32_t)nchild++;
    if ((int)slot >= C.capacity) {
      count(F.Y, kCntChildOverflow);
      return;
    }
    C.x[slot] = x; C.y[slot] = y; C.z[slot] = z;
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
    const int icont = inside_mesh(i, j, k) ? F.M.contact[cell_index(i, j, k)] - 1 : -1;
    if (with_current) {
      if (idir == kRight) tally_add_i64(F.Y.rcurrent + jc + 1, charge, kChargeScale);
      if (idir == kLeft) tally_add_i64(F.Y.lcurrent + jc, charge, kChargeScale);
    }
    if (icont >= 0 && icont < kMaxContacts) {
      atomicAdd(reinterpret_cast<unsigned long long *>(F.Y.contact + icont * 6 + 3), 1ull);
      contact_add(icont, 4, charge, kChargeScale);
      contact_add(icont, 2, energy, kEnergyScale);  // the reference adds to EnergyGen here (src/CellHit.cpp:542)
    }
  }
  __device__ void load_cell_fields() {
    const int c = cell_index();
    Rho = F.M.rho[c];
    DA = F.M.da[c];
    const double *f = (type == 0 ? F.M.efield : F.M.hfield) + 3 * (size_t)c;
    Ex = f[0];
    Ey = f[1];
    Ez = f[2];
  }
  // HitCell, src/CellHit.cpp:96-211.  Returns false when the particle would
  // leave the device through a PASS / GENERATE face on the outer y boundary.
  __device__ bool HitCell() {
    const int imot = F.M.motion[(size_t)cell_index() * 6 + idir];
    if (imot == kPass || imot == kGenerate || imot == kGenRef) {
      if ((idir == kLeft && jc == 0) || (idir == kRight && jc == F.M.ny - 1)) return false;
    }
    if (imot == kPass) Pass();
    else if (imot == kReflect) Reflect();
    else if (imot == kScattOx) {
      if (F.M.surface_scatter) Reflect();
      else {
        if (Random() > F.T.difpr[type]) Reflect();
        else Diffuse();
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
      count(F.Y, kCntNoTet);
    }
    load_cell_fields();
    return true;
  }
  // ParticleSurfaceScatter, src/ParSurfaceScatter.cpp:48-61, with the
  // surface-phonon branches' drand defined (see file note).
  __device__ void ParticleSurfaceScatter() {
    if (Random() * surf_gamma < rough_rate) {
      idir = F.M.surface_dir[min(max(F.M.nearest_surf[cell_index()], 0), kMaxSurfaces - 1)];
      Diffuse();
      return;
    }
    self = false;
    if (type == 0) {
      const double drand = Random() * electron_rate_sum();
      const int iscat = pick_electron_mechanism(drand);
      if (iscat < 0) { self = true; return; }
      if (((iscat % F.T.scpre) + 1) == F.T.scpre) ESCATII(iscat);
      else EPSCAT(iscat);
    } else {
      const double drand = Random() * hole_rate_sum();
      const int iscat = pick_hole_mechanism(drand);
      if (iscat < 0) { self = true; return; }
      if (((iscat % F.T.scprh) + 1) == F.T.scprh) HSCATII(iscat);
      else HPSCAT(iscat);
    }
  }

  // One particle, one step: particle_fly, src/mcmodel.cpp:1874-2161.
  // Returns 0 done, 1 caught, 2 unfinished (outer-boundary PASS).
  __device__ int fly() {
    catch_ = false;
    bool get_tet = true, get_cell = true, get_ph = true, get_imp = true, get_surf = true;
    double ssnl = 0, imprnl = 0, phrnl = 0;
    double TetTf = 0, CellTf = 0, PhScTf, ImpScTf, SurfScTf, Tf;
    bool too_far = false;
    load_cell_fields();
    iband = F.T.ibt[itet];
    GetV();
    int loop = 0;
    const double dt = F.dt;
    surf_gamma = 0;
    imp_gamma = 0;
    while (left_time > 0) {
      GetV();
      if (++loop > kMaxEvents) {
        count(F.Y, kCntTooManyEvents);
        catch_ = true;
        break;
      }
      if (get_tet) { TetTf = TetTime(); get_tet = false; }
      if (get_cell) { CellTf = CellTime(); get_cell = false; }
      if (get_ph) { phrnl = -log(Random()); get_ph = false; }
      const double g = F.T.gamtet[itet];
      PhScTf = phrnl / g;
      if (iband == F.T.bandof[0]) {
        if (get_imp) { imprnl = -log(Random()); get_imp = false; }
        imp_gamma = GetImpScGamma();
        ImpScTf = imprnl / imp_gamma;
      } else {
        ImpScTf = 2 * dt;
        imp_gamma = 1.0 / F.T.scrt0;
      }
      if (F.M.surface_scatter && F.M.in_surf[cell_index()]) {
        if (get_surf) { ssnl = -log(Random()); get_surf = false; }
        GetSurfScRate();
        SurfScTf = (surf_gamma > 0 && ssnl > 0) ? ssnl / surf_gamma : 2 * dt;
      } else {
        SurfScTf = 2 * dt;
      }
      // Min(..., flag), src/Constant_GlobalVariable_MathFunction.cpp:92-118
      int flag = 1;
      Tf = TetTf;
      if (Tf > CellTf) { Tf = CellTf; flag = 2; }
      if (Tf > PhScTf) { Tf = PhScTf; flag = 3; }
      if (Tf > ImpScTf) { Tf = ImpScTf; flag = 4; }
      if (Tf > SurfScTf) { Tf = SurfScTf; flag = 5; }
      if (Tf > left_time) { Tf = left_time; flag = 6; }
      if (Tf < kMyZero) {
        catch_ = true;
        break;
      }
      TetTf -= Tf;
      CellTf -= Tf;
      PhScTf -= Tf;
      ImpScTf -= Tf;
      SurfScTf -= Tf;
      left_time -= Tf;
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
        break;
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
          if (type == 0) ElectronPhononScatter();
          else HolePhononScatter();
          if (!self) {
            get_tet = true;
            get_cell = true;
            count(F.Y, kCntPhonon);
          }
          get_ph = true;
          break;
        case 4:
          if (type == 0) ElectronImpurityScatter();
          if (!self) {
            get_tet = true;
            get_cell = true;
            count(F.Y, kCntImpurity);
          }
          get_imp = true;
          break;
        case 5:
          ParticleSurfaceScatter();
          if (!self) {
            get_tet = true;
            get_cell = true;
          }
          get_surf = true;
          break;
      }
      if (too_far || catch_) break;
    }
    atomicAdd(&F.Y.counters[kCntEvents], (unsigned long long)loop);
    if (catch_) {
      count(F.Y, kCntCaught);
      return 1;
    }
    if (too_far) {
      count(F.Y, kCntUnfinished);
      return 2;
    }
    return 0;
  }
};

}  // namespace mcb200
