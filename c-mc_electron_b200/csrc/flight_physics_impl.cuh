// flight_physics_impl.cuh -- out-of-line members of Flyer (flight_physics.cuh).
#pragma once

#include "flight_physics.cuh"

namespace mcb200 {

__device__ __forceinline__ double dfii(double x1, double y1, double z1, double x2, double y2, double z2, double x3,
                                       double y3, double z3) {
  // Band::FII, src/Band.cpp:335-353
  const double sbx = (y2 - y1) * (z3 - z1) - (y3 - y1) * (z2 - z1);
  const double sby = (x3 - x1) * (z2 - z1) - (x2 - x1) * (z3 - z1);
  const double sbz = (x2 - x1) * (y3 - y1) - (x3 - x1) * (y2 - y1);
  return 0.50 * sqrt(sbx * sbx + sby * sby + sbz * sbz);
}

// Band::SURF, src/Band.cpp:194-332.
__device__ double Flyer::SURF(double eps, int it) const {
  const int4 nd = F.T.tnode[it];
  const double4 k0 = F.T.knode[nd.x], k1 = F.T.knode[nd.y], k2 = F.T.knode[nd.z], k3 = F.T.knode[nd.w];
  const double e0 = k0.w, e1 = k1.w, e2 = k2.w, e3 = k3.w;
  if (!(eps > e0 && eps < e3)) return 0.0;
  auto rel = [&](const double4 &p, const double4 &q, double &ox, double &oy, double &oz) {
    const double r = (eps - p.w) / (q.w - p.w);
    ox = r * (q.x - p.x);
    oy = r * (q.y - p.y);
    oz = r * (q.z - p.z);
  };
  auto abs_ = [&](const double4 &p, const double4 &q, double &ox, double &oy, double &oz) {
    const double r = (eps - p.w) / (q.w - p.w);
    ox = r * (q.x - p.x) + p.x;
    oy = r * (q.y - p.y) + p.y;
    oz = r * (q.z - p.z) + p.z;
  };
  double ax, ay, az, bx, by, bz, cx, cy, cz, dx, dy, dz;
  if (eps <= e1) {
    rel(k0, k1, ax, ay, az);
    rel(k0, k2, bx, by, bz);
    rel(k0, k3, cx, cy, cz);
    return dfii(ax, ay, az, bx, by, bz, cx, cy, cz);
  }
  if (eps > e1 && eps < e2) {
    abs_(k0, k2, ax, ay, az);
    abs_(k1, k2, bx, by, bz);
    abs_(k0, k3, cx, cy, cz);
    abs_(k1, k3, dx, dy, dz);
    const double a1 = dfii(ax, ay, az, bx, by, bz, cx, cy, cz);
    const double a2 = dfii(dx, dy, dz, bx, by, bz, cx, cy, cz);
    const double a3 = dfii(ax, ay, az, dx, dy, dz, cx, cy, cz);
    const double a4 = dfii(ax, ay, az, bx, by, bz, dx, dy, dz);
    return 0.50 * (a1 + a2 + a3 + a4);
  }
  if (eps > e2 && eps < e3) {
    rel(k3, k0, ax, ay, az);
    rel(k3, k1, bx, by, bz);
    rel(k3, k2, cx, cy, cz);
    return dfii(ax, ay, az, bx, by, bz, cx, cy, cz);
  }
  return 0.0;
}

// getK, src/ParticleUtils.cpp:122-284.
__device__ void Flyer::getK() {
  const double rv1 = 1.0 - sqrt(Random());
  const double rv2 = Random() * (1.0 - rv1);
  const int4 nd = F.T.tnode[itet];
  const double4 k0 = F.T.knode[nd.x], k1 = F.T.knode[nd.y], k2 = F.T.knode[nd.z], k3 = F.T.knode[nd.w];
  if ((energy < k0.w) || (energy > k3.w)) energy = k0.w + (k3.w - k0.w) * Random();
  double xkl, ykl, zkl;
  if (energy <= k1.w) {
    double r = (energy - k0.w) / (k1.w - k0.w);
    const double ax = r * (k1.x - k0.x), ay = r * (k1.y - k0.y), az = r * (k1.z - k0.z);
    r = (energy - k0.w) / (k2.w - k0.w);
    const double bx = r * (k2.x - k0.x), by = r * (k2.y - k0.y), bz = r * (k2.z - k0.z);
    r = (energy - k0.w) / (k3.w - k0.w);
    const double cx = r * (k3.x - k0.x), cy = r * (k3.y - k0.y), cz = r * (k3.z - k0.z);
    xkl = rv1 * (bx - ax) + rv2 * (cx - ax) + ax + k0.x;
    ykl = rv1 * (by - ay) + rv2 * (cy - ay) + ay + k0.y;
    zkl = rv1 * (bz - az) + rv2 * (cz - az) + az + k0.z;
  } else if (energy < k2.w) {
    double r = (energy - k0.w) / (k2.w - k0.w);
    const double ax = r * (k2.x - k0.x) + k0.x, ay = r * (k2.y - k0.y) + k0.y, az = r * (k2.z - k0.z) + k0.z;
    r = (energy - k1.w) / (k2.w - k1.w);
    const double bx = r * (k2.x - k1.x) + k1.x, by = r * (k2.y - k1.y) + k1.y, bz = r * (k2.z - k1.z) + k1.z;
    r = (energy - k0.w) / (k3.w - k0.w);
    const double cx = r * (k3.x - k0.x) + k0.x, cy = r * (k3.y - k0.y) + k0.y, cz = r * (k3.z - k0.z) + k0.z;
    r = (energy - k1.w) / (k3.w - k1.w);
    const double dx = r * (k3.x - k1.x) + k1.x, dy = r * (k3.y - k1.y) + k1.y, dz = r * (k3.z - k1.z) + k1.z;
    const double a1 = dfii(ax, ay, az, bx, by, bz, cx, cy, cz);
    const double a2 = dfii(dx, dy, dz, bx, by, bz, cx, cy, cz);
    const double a3 = dfii(ax, ay, az, dx, dy, dz, cx, cy, cz);
    const double a4 = dfii(ax, ay, az, bx, by, bz, dx, dy, dz);
    const double ar = Random() * (a1 + a2 + a3 + a4);
    if (ar < a1) {
      xkl = rv1 * (bx - ax) + rv2 * (cx - ax) + ax;
      ykl = rv1 * (by - ay) + rv2 * (cy - ay) + ay;
      zkl = rv1 * (bz - az) + rv2 * (cz - az) + az;
    } else if (ar < (a1 + a2)) {
      xkl = rv1 * (bx - dx) + rv2 * (cx - dx) + dx;
      ykl = rv1 * (by - dy) + rv2 * (cy - dy) + dy;
      zkl = rv1 * (bz - dz) + rv2 * (cz - dz) + dz;
    } else if (ar < (a1 + a2 + a3)) {
      xkl = rv1 * (dx - ax) + rv2 * (cx - ax) + ax;
      ykl = rv1 * (dy - ay) + rv2 * (cy - ay) + ay;
      zkl = rv1 * (dz - az) + rv2 * (cz - az) + az;
    } else {
      xkl = rv1 * (bx - ax) + rv2 * (dx - ax) + ax;
      ykl = rv1 * (by - ay) + rv2 * (dy - ay) + ay;
      zkl = rv1 * (bz - az) + rv2 * (dz - az) + az;
    }
  } else {
    double r = (energy - k3.w) / (k0.w - k3.w);
    const double ax = r * (k0.x - k3.x), ay = r * (k0.y - k3.y), az = r * (k0.z - k3.z);
    r = (energy - k3.w) / (k1.w - k3.w);
    const double bx = r * (k1.x - k3.x), by = r * (k1.y - k3.y), bz = r * (k1.z - k3.z);
    r = (energy - k3.w) / (k2.w - k3.w);
    const double cx = r * (k2.x - k3.x), cy = r * (k2.y - k3.y), cz = r * (k2.z - k3.z);
    xkl = rv1 * (bx - ax) + rv2 * (cx - ax) + ax + k3.x;
    ykl = rv1 * (by - ay) + rv2 * (cy - ay) + ay + k3.y;
    zkl = rv1 * (bz - az) + rv2 * (cz - az) + az + k3.z;
  }
  out_wedge(kx, ky, kz, xkl, ykl, zkl);
}

// Interpolation weight of the energy tables (CALSCATTE / CALSCATTH prologue).
struct TabPos {
  int mode;  // 0: below table, 1: above, 2: interior
  int itab;
  double intp;
};
__device__ __forceinline__ TabPos tab_pos(const DevTables &T, double eed) {
  TabPos p;
  if (eed <= 0.0) { p.mode = 0; p.itab = 0; p.intp = 0; }
  else if (eed >= T.emax) { p.mode = 1; p.itab = kNT - 1; p.intp = 0; }
  else {
    p.mode = 2;
    p.itab = min((int)(eed / T.dtable), kNT - 2);
    p.intp = (eed - T.energy[p.itab]) / (T.energy[p.itab + 1] - T.energy[p.itab]);
  }
  return p;
}
__device__ __forceinline__ double tab_at(const double *tab, const TabPos &p) {
  if (p.mode != 2) return tab[p.itab];
  return tab[p.itab] + p.intp * (tab[p.itab + 1] - tab[p.itab]);
}
__device__ __forceinline__ double tab_at_strided(const double *tab, int stride, const TabPos &p) {
  if (p.mode != 2) return tab[(size_t)p.itab * stride];
  const double a = tab[(size_t)p.itab * stride], b = tab[(size_t)(p.itab + 1) * stride];
  return a + p.intp * (b - a);
}

// Entry idx of Band::CALSCATTE (src/Band.cpp:2165-2231) for initial band ib.
__device__ __forceinline__ double electron_rate(const DevTables &T, const TabPos &p, int ini, int idx) {
  const int f = idx / T.scpre, is = idx % T.scpre;
  if (is < T.scpre - 1)
    return T.scatte[(is * 4 + f) * 4 + ini] * tab_at(T.dose + (size_t)(is * 4 + f) * kNT, p);
  return tab_at(T.scattiie + (size_t)(f * 4 + ini) * kNT, p);
}
// Entry idx of Band::CALSCATTH (src/Band.cpp:2098-2162).
__device__ __forceinline__ double hole_rate(const DevTables &T, const TabPos &p, int ini, int idx) {
  const int f = idx / T.scprh, is = idx % T.scprh;
  if (is < T.scprh - 1)
    return T.scatth[(is * 3 + f) * 3 + ini] * tab_at(T.dosh + (size_t)(is * 3 + f) * kNT, p);
  return tab_at(T.scattiih + (size_t)(f * 3 + ini) * kNT, p);
}

// Mechanism search of ElectronPhononScatter, src/ElectronPhononScatter.cpp:47-63.
__device__ int Flyer::pick_electron_mechanism(double drand) const {
  const TabPos p = tab_pos(F.T, energy);
  const int ini = iband - F.T.bandof[0], n = F.T.scpre * F.T.nband[0];
  int iscat = -1;
  double dscat = 0.0;
  while (drand > dscat) {
    iscat = iscat + 1;
    if (iscat >= n) return -1;
    dscat = dscat + electron_rate(F.T, p, ini, iscat);
  }
  return iscat;
}
__device__ double Flyer::electron_rate_sum() const {
  const TabPos p = tab_pos(F.T, energy);
  const int ini = iband - F.T.bandof[0], n = F.T.scpre * F.T.nband[0];
  double s = 0.0;
  for (int i = 0; i < n; ++i) s += electron_rate(F.T, p, ini, i);
  return s;
}
// Mechanism search of HolePhononScatter, src/HolePhononScatter.cpp:49-66.
__device__ int Flyer::pick_hole_mechanism(double drand) const {
  const TabPos p = tab_pos(F.T, energy);
  const int ini = iband - F.T.bandof[1], n = F.T.scprh * F.T.nband[1];
  int iscat = -1;
  double dscat = 0.0;
  while (drand > dscat) {
    iscat = iscat + 1;
    if (iscat >= n) return -1;
    dscat = dscat + hole_rate(F.T, p, ini, iscat);
  }
  return iscat;
}
__device__ double Flyer::hole_rate_sum() const {
  const TabPos p = tab_pos(F.T, energy);
  const int ini = iband - F.T.bandof[1], n = F.T.scprh * F.T.nband[1];
  double s = 0.0;
  for (int i = 0; i < n; ++i) s += hole_rate(F.T, p, ini, i);
  return s;
}

// EleImpScUpdateK, src/ElectronImpurityScatter.cpp:188-306: Brooks-Herring
// final state in the ellipsoidal-valley picture, accepted by rejection.
__device__ void Flyer::EleImpScUpdateK() {
  const DevTables &T = F.T;
  double xkl, ykl, zkl;
  in_wedge(xkl, ykl, zkl, kx, ky, kz);
  xkl = xkl - 0.85 * T.a0pi;
  xkl = xkl * sqrt(T.meld / T.mell);
  ykl = ykl * sqrt(T.meld / T.melt);
  zkl = zkl * sqrt(T.meld / T.melt);
  const double betaq = T.frickel * 4 * kPiD * Rho / T.eps_si;
  const double eebeta = betaq / (2.0 * T.meld);
  const double alfa = eebeta * T.meld / (2.0 * energy * T.melt);
  double pr = Random() / (1.0 + 0.5 * alfa);
  const double costr = 1.0 - alfa * pr / (1.0 - pr);
  const double sintr = sqrt(1.0 - costr * costr);
  pr = 2.0 * kPiD * Random();
  const double cospr = cos(pr), sinpr = sin(pr);
  const double ca = sqrt(xkl * xkl + ykl * ykl);
  const double cb = sqrt(ca * ca + zkl * zkl);
  const double xkll = cb * sintr * cospr, ykll = cb * sintr * sinpr, zkll = cb * costr;
  const double cosphi = xkl / ca, sinphi = ykl / ca, costheta = zkl / cb, sintheta = ca / cb;
  const double xklll = cosphi * costheta * xkll - sinphi * ykll + cosphi * sintheta * zkll;
  const double yklll = sinphi * costheta * xkll + cosphi * ykll + sinphi * sintheta * zkll;
  const double zklll = -sintheta * xkll + costheta * zkll;
  const double dx = xkl - xklll, dy = ykl - yklll, dz = zkl - zklll;
  const double dn = pow(betaq + T.mell / T.meld * dx * dx + T.melt / T.meld * (dy * dy + dz * dz), -2.0);
  const double dnmax = pow(betaq + T.melt / T.meld * dx * dx + T.melt / T.meld * (dy * dy + dz * dz), -2.0);
  if (dn > Random() * dnmax) {
    xkl = xklll * sqrt(T.mell / T.meld);
    ykl = yklll * sqrt(T.melt / T.meld);
    zkl = zklll * sqrt(T.melt / T.meld);
    xkl = xkl + 0.85 * T.a0pi;
    out_wedge(kx, ky, kz, xkl, ykl, zkl);
    CONFBZ(kx, ky, kz);
    Getisym();
    GetEnergy();
    self = false;
  } else {
    self = true;
  }
}

// Diffuse, src/CellHit.cpp:243-386: random state on the iso-energy surface,
// then mirrored so the velocity points back into the device.
__device__ void Flyer::Diffuse() {
  const int ibandold = iband, itetold = itet, isymold = isym;
  const double xkold = kx, ykold = ky, zkold = kz;
  TALIND(1);
  get_state();
  auto restore = [&]() {
    iband = ibandold; itet = itetold; isym = isymold;
    kx = xkold; ky = ykold; kz = zkold;
  };
  if (self) restore();
  GetV();
  switch (idir) {
    case kUp:
      if (vx == 0.0) restore();
      if (vx < 0.0) reflect_axis(0);
      break;
    case kRight:
      if (vy == 0.0) restore();
      if (vy > 0.0) reflect_axis(1);
      break;
    case kDown:
      if (vx == 0.0) restore();
      if (vx > 0.0) reflect_axis(0);
      break;
    case kLeft:
      if (vy == 0.0) restore();
      if (vy < 0.0) reflect_axis(1);
      break;
    case kFront:
      if (vz == 0.0) restore();
      if (vz < 0.0) reflect_axis(2);
      break;
    case kBack:
      if (vz == 0.0) restore();
      if (vz > 0.0) reflect_axis(2);
      break;
  }
}

}  // namespace mcb200
