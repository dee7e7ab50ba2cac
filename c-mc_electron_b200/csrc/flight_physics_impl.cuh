// flight_physics_impl.cuh -- out-of-line members of FlyerT (flight_physics.cuh).
#pragma once

#include "flight_physics.cuh"

namespace mcb200 {

template <typename R>
__device__ __forceinline__ R dfii(R x1, R y1, R z1, R x2, R y2, R z2, R x3, R y3, R z3) {
  // Band::FII, src/Band.cpp:335-353
  const R sbx = (y2 - y1) * (z3 - z1) - (y3 - y1) * (z2 - z1);
  const R sby = (x3 - x1) * (z2 - z1) - (x2 - x1) * (z3 - z1);
  const R sbz = (x2 - x1) * (y3 - y1) - (x3 - x1) * (y2 - y1);
  return (R)0.50 * m_sqrt(sbx * sbx + sby * sby + sbz * sbz);
}

// Band::SURF, src/Band.cpp:194-332.
template <typename R>
__device__ R FlyerT<R>::SURF(R eps, int it) const {
  const int4 nd = F.T.tnode[it];
  const V4 *kn = TB::knode(F.T);
  const V4 k0 = kn[nd.x], k1 = kn[nd.y], k2 = kn[nd.z], k3 = kn[nd.w];
  const R e0 = k0.w, e1 = k1.w, e2 = k2.w, e3 = k3.w;
  if (!(eps > e0 && eps < e3)) return 0;
  auto rel = [&](const V4 &p, const V4 &q, R &ox, R &oy, R &oz) {
    const R r = (eps - p.w) / (q.w - p.w);
    ox = r * (q.x - p.x);
    oy = r * (q.y - p.y);
    oz = r * (q.z - p.z);
  };
  auto abs_ = [&](const V4 &p, const V4 &q, R &ox, R &oy, R &oz) {
    const R r = (eps - p.w) / (q.w - p.w);
    ox = r * (q.x - p.x) + p.x;
    oy = r * (q.y - p.y) + p.y;
    oz = r * (q.z - p.z) + p.z;
  };
  R ax, ay, az, bx, by, bz, cx, cy, cz, dx, dy, dz;
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
    const R a1 = dfii(ax, ay, az, bx, by, bz, cx, cy, cz);
    const R a2 = dfii(dx, dy, dz, bx, by, bz, cx, cy, cz);
    const R a3 = dfii(ax, ay, az, dx, dy, dz, cx, cy, cz);
    const R a4 = dfii(ax, ay, az, bx, by, bz, dx, dy, dz);
    return (R)0.50 * (a1 + a2 + a3 + a4);
  }
  if (eps > e2 && eps < e3) {
    rel(k3, k0, ax, ay, az);
    rel(k3, k1, bx, by, bz);
    rel(k3, k2, cx, cy, cz);
    return dfii(ax, ay, az, bx, by, bz, cx, cy, cz);
  }
  return 0;
}

// getK, src/ParticleUtils.cpp:122-284.
template <typename R>
__device__ void FlyerT<R>::getK() {
  const R rv1 = (R)1.0 - m_sqrt(Random());
  const R rv2 = Random() * ((R)1.0 - rv1);
  const int4 nd = F.T.tnode[itet];
  const V4 *kn = TB::knode(F.T);
  const V4 k0 = kn[nd.x], k1 = kn[nd.y], k2 = kn[nd.z], k3 = kn[nd.w];
  R e = (R)energy;
  if ((e < k0.w) || (e > k3.w)) {
    e = k0.w + (k3.w - k0.w) * Random();
    energy = e;
  }
  R xkl, ykl, zkl;
  if (e <= k1.w) {
    R r = (e - k0.w) / (k1.w - k0.w);
    const R ax = r * (k1.x - k0.x), ay = r * (k1.y - k0.y), az = r * (k1.z - k0.z);
    r = (e - k0.w) / (k2.w - k0.w);
    const R bx = r * (k2.x - k0.x), by = r * (k2.y - k0.y), bz = r * (k2.z - k0.z);
    r = (e - k0.w) / (k3.w - k0.w);
    const R cx = r * (k3.x - k0.x), cy = r * (k3.y - k0.y), cz = r * (k3.z - k0.z);
    xkl = rv1 * (bx - ax) + rv2 * (cx - ax) + ax + k0.x;
    ykl = rv1 * (by - ay) + rv2 * (cy - ay) + ay + k0.y;
    zkl = rv1 * (bz - az) + rv2 * (cz - az) + az + k0.z;
  } else if (e < k2.w) {
    R r = (e - k0.w) / (k2.w - k0.w);
    const R ax = r * (k2.x - k0.x) + k0.x, ay = r * (k2.y - k0.y) + k0.y, az = r * (k2.z - k0.z) + k0.z;
    r = (e - k1.w) / (k2.w - k1.w);
    const R bx = r * (k2.x - k1.x) + k1.x, by = r * (k2.y - k1.y) + k1.y, bz = r * (k2.z - k1.z) + k1.z;
    r = (e - k0.w) / (k3.w - k0.w);
    const R cx = r * (k3.x - k0.x) + k0.x, cy = r * (k3.y - k0.y) + k0.y, cz = r * (k3.z - k0.z) + k0.z;
    r = (e - k1.w) / (k3.w - k1.w);
    const R dx = r * (k3.x - k1.x) + k1.x, dy = r * (k3.y - k1.y) + k1.y, dz = r * (k3.z - k1.z) + k1.z;
    const R a1 = dfii(ax, ay, az, bx, by, bz, cx, cy, cz);
    const R a2 = dfii(dx, dy, dz, bx, by, bz, cx, cy, cz);
    const R a3 = dfii(ax, ay, az, dx, dy, dz, cx, cy, cz);
    const R a4 = dfii(ax, ay, az, bx, by, bz, dx, dy, dz);
    const R ar = Random() * (a1 + a2 + a3 + a4);
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
    R r = (e - k3.w) / (k0.w - k3.w);
    const R ax = r * (k0.x - k3.x), ay = r * (k0.y - k3.y), az = r * (k0.z - k3.z);
    r = (e - k3.w) / (k1.w - k3.w);
    const R bx = r * (k1.x - k3.x), by = r * (k1.y - k3.y), bz = r * (k1.z - k3.z);
    r = (e - k3.w) / (k2.w - k3.w);
    const R cx = r * (k2.x - k3.x), cy = r * (k2.y - k3.y), cz = r * (k2.z - k3.z);
    xkl = rv1 * (bx - ax) + rv2 * (cx - ax) + ax + k3.x;
    ykl = rv1 * (by - ay) + rv2 * (cy - ay) + ay + k3.y;
    zkl = rv1 * (bz - az) + rv2 * (cz - az) + az + k3.z;
  }
  out_wedge(kx, ky, kz, xkl, ykl, zkl);
}

// Interpolation weight of the energy tables (CALSCATTE / CALSCATTH prologue).
template <typename R>
struct TabPosT {
  int mode;  // 0: below table, 1: above, 2: interior
  int itab;
  R intp;
};
using TabPos = TabPosT<double>;
template <typename R>
__device__ __forceinline__ TabPosT<R> tab_pos(const DevTables &T, R eed) {
  TabPosT<R> p;
  const R *E = Tab<R>::energy(T);
  if (eed <= (R)0) { p.mode = 0; p.itab = 0; p.intp = 0; }
  else if (eed >= (R)T.emax) { p.mode = 1; p.itab = kNT - 1; p.intp = 0; }
  else {
    p.mode = 2;
    p.itab = min((int)(eed / (R)T.dtable), kNT - 2);
    p.intp = (eed - E[p.itab]) / (E[p.itab + 1] - E[p.itab]);
  }
  return p;
}
template <typename R>
__device__ __forceinline__ R tab_at(const R *tab, const TabPosT<R> &p) {
  if (p.mode != 2) return tab[p.itab];
  return tab[p.itab] + p.intp * (tab[p.itab + 1] - tab[p.itab]);
}
template <typename R>
__device__ __forceinline__ R tab_at_strided(const R *tab, int stride, const TabPosT<R> &p) {
  if (p.mode != 2) return tab[(size_t)p.itab * stride];
  const R a = tab[(size_t)p.itab * stride], b = tab[(size_t)(p.itab + 1) * stride];
  return a + p.intp * (b - a);
}

// Entry idx of Band::CALSCATTE (src/Band.cpp:2165-2231) for initial band ib.
template <typename R>
__device__ __forceinline__ R electron_rate(const DevTables &T, const TabPosT<R> &p, int ini, int idx) {
  const int f = idx / T.scpre, is = idx % T.scpre;
  if (is < T.scpre - 1)
    return Tab<R>::scatte(T)[(is * 4 + f) * 4 + ini] * tab_at(Tab<R>::dose(T) + (size_t)(is * 4 + f) * kNT, p);
  return tab_at(Tab<R>::scattiie(T) + (size_t)(f * 4 + ini) * kNT, p);
}
// Entry idx of Band::CALSCATTH (src/Band.cpp:2098-2162).
template <typename R>
__device__ __forceinline__ R hole_rate(const DevTables &T, const TabPosT<R> &p, int ini, int idx) {
  const int f = idx / T.scprh, is = idx % T.scprh;
  if (is < T.scprh - 1)
    return Tab<R>::scatth(T)[(is * 3 + f) * 3 + ini] * tab_at(Tab<R>::dosh(T) + (size_t)(is * 3 + f) * kNT, p);
  return tab_at(Tab<R>::scattiih(T) + (size_t)(f * 3 + ini) * kNT, p);
}

// Mechanism search of ElectronPhononScatter, src/ElectronPhononScatter.cpp:47-63.
template <typename R>
__device__ int FlyerT<R>::pick_electron_mechanism(R drand) const {
  const TabPosT<R> p = tab_pos(F.T, (R)energy);
  const int ini = iband - F.T.bandof[0], n = F.T.scpre * F.T.nband[0];
  int iscat = -1;
  R dscat = 0;
  while (drand > dscat) {
    iscat = iscat + 1;
    if (iscat >= n) return -1;
    dscat = dscat + electron_rate(F.T, p, ini, iscat);
  }
  return iscat;
}
template <typename R>
__device__ R FlyerT<R>::electron_rate_sum() const {
  const TabPosT<R> p = tab_pos(F.T, (R)energy);
  const int ini = iband - F.T.bandof[0], n = F.T.scpre * F.T.nband[0];
  R s = 0;
  for (int i = 0; i < n; ++i) s += electron_rate(F.T, p, ini, i);
  return s;
}
// Mechanism search of HolePhononScatter, src/HolePhononScatter.cpp:49-66.
template <typename R>
__device__ int FlyerT<R>::pick_hole_mechanism(R drand) const {
  const TabPosT<R> p = tab_pos(F.T, (R)energy);
  const int ini = iband - F.T.bandof[1], n = F.T.scprh * F.T.nband[1];
  int iscat = -1;
  R dscat = 0;
  while (drand > dscat) {
    iscat = iscat + 1;
    if (iscat >= n) return -1;
    dscat = dscat + hole_rate(F.T, p, ini, iscat);
  }
  return iscat;
}
template <typename R>
__device__ R FlyerT<R>::hole_rate_sum() const {
  const TabPosT<R> p = tab_pos(F.T, (R)energy);
  const int ini = iband - F.T.bandof[1], n = F.T.scprh * F.T.nband[1];
  R s = 0;
  for (int i = 0; i < n; ++i) s += hole_rate(F.T, p, ini, i);
  return s;
}

// EleImpScUpdateK, src/ElectronImpurityScatter.cpp:188-306: Brooks-Herring
// final state in the ellipsoidal-valley picture, accepted by rejection.
// FP64 keeps the reference's pow(., -2.0); FP32 writes it as 1 / q^2.
template <typename R>
__device__ void FlyerT<R>::EleImpScUpdateK() {
  const DevTables &T = F.T;
  R xkl, ykl, zkl;
  in_wedge(xkl, ykl, zkl, kx, ky, kz);
  xkl = xkl - (R)0.85 * (R)T.a0pi;
  xkl = xkl * m_sqrt((R)(T.meld / T.mell));
  ykl = ykl * m_sqrt((R)(T.meld / T.melt));
  zkl = zkl * m_sqrt((R)(T.meld / T.melt));
  R betaq;
  if constexpr (sizeof(R) == 4) betaq = imp_beta;
  else betaq = T.frickel * 4 * kPiD * Rho / T.eps_si;
  const R eebeta = betaq / (R)(2.0 * T.meld);
  const R alfa = eebeta * (R)T.meld / ((R)2.0 * (R)energy * (R)T.melt);
  R pr = Random() / ((R)1.0 + (R)0.5 * alfa);
  const R costr = (R)1.0 - alfa * pr / ((R)1.0 - pr);
  const R sintr = m_sqrt((R)1.0 - costr * costr);
  pr = (R)(2.0 * kPiD) * Random();
  R cospr, sinpr;
  m_sincos(pr, &sinpr, &cospr);
  const R ca = m_sqrt(xkl * xkl + ykl * ykl);
  const R cb = m_sqrt(ca * ca + zkl * zkl);
  const R xkll = cb * sintr * cospr, ykll = cb * sintr * sinpr, zkll = cb * costr;
  const R cosphi = xkl / ca, sinphi = ykl / ca, costheta = zkl / cb, sintheta = ca / cb;
  const R xklll = cosphi * costheta * xkll - sinphi * ykll + cosphi * sintheta * zkll;
  const R yklll = sinphi * costheta * xkll + cosphi * ykll + sinphi * sintheta * zkll;
  const R zklll = -sintheta * xkll + costheta * zkll;
  const R dx = xkl - xklll, dy = ykl - yklll, dz = zkl - zklll;
  const R ml = (R)(T.mell / T.meld), mt = (R)(T.melt / T.meld);
  const R q = betaq + ml * dx * dx + mt * (dy * dy + dz * dz);
  const R qmax = betaq + mt * dx * dx + mt * (dy * dy + dz * dz);
  R dn, dnmax;
  if constexpr (sizeof(R) == 4) {
    dn = (R)1 / (q * q);
    dnmax = (R)1 / (qmax * qmax);
  } else {
    dn = pow(q, -2.0);
    dnmax = pow(qmax, -2.0);
  }
  if (dn > Random() * dnmax) {
    xkl = xklll * m_sqrt((R)(T.mell / T.meld));
    ykl = yklll * m_sqrt((R)(T.melt / T.meld));
    zkl = zklll * m_sqrt((R)(T.melt / T.meld));
    xkl = xkl + (R)0.85 * (R)T.a0pi;
    out_wedge(kx, ky, kz, xkl, ykl, zkl);
    CONFBZ(kx, ky, kz);
    loc_mode = kLocImpurity;  // Getisym + GetEnergy in run_locate
    self = false;
  } else {
    self = true;
  }
}

}  // namespace mcb200
