// mg_setup.cpp -- Galerkin multigrid hierarchy (see mg_setup.h).
#include "mg_setup.h"

#include <algorithm>
#include <cmath>
#include <stdexcept>

namespace mcb200 {
namespace {

// Coarse nodes of one axis: the first and last node are kept; an interior
// node is dropped when the interval it splits is no wider than `h` and its
// predecessor was kept, so no two consecutive nodes are dropped (every
// coarse coupling stays within one coarse node per axis).  With `h` twice
// the finest spacing of the level, finely spaced regions coarsen first and
// coarse regions wait until the mesh around them has caught up, which
// coarsens anisotropic cells along their short sides only.
std::vector<int> select_axis(const std::vector<double> &x, double h) {
  const int n = (int)x.size();
  std::vector<int> keep{0};
  int i = 0;
  while (i < n - 1) {
    if (i + 2 <= n - 1 && x[i + 2] - x[i] <= h) i += 2;
    else i += 1;
    keep.push_back(i);
  }
  return keep;
}

MgAxis make_axis(const std::vector<double> &x, const std::vector<int> &keep) {
  const int n = (int)x.size();
  MgAxis a;
  a.c0.resize(n); a.c1.resize(n); a.w0.resize(n); a.w1.resize(n);
  int c = 0;
  for (int i = 0; i < n; ++i) {
    while (c + 1 < (int)keep.size() && keep[c + 1] <= i) ++c;
    int c0 = c, c1 = c;
    double w1 = 0.0;
    if (keep[c] != i) {
      c1 = c + 1;
      const double xa = x[keep[c0]], xb = x[keep[c1]];
      w1 = (x[i] - xa) / (xb - xa);
    }
    a.c0[i] = c0; a.c1[i] = c1; a.w0[i] = 1.0 - w1; a.w1[i] = w1;
  }
  return a;
}

// Weight of coarse node c in the interpolation of fine index i.
double tap(const MgAxis &a, int i, int c) {
  double v = 0.0;
  if (a.c0[i] == c) v += a.w0[i];
  if (a.c1[i] == c && a.c1[i] != a.c0[i]) v += a.w1[i];
  return v;
}

std::vector<double> restriction_taps(const MgAxis &a, const std::vector<int> &keep) {
  const int n = (int)a.c0.size();
  std::vector<double> r(3 * keep.size(), 0.0);
  for (size_t c = 0; c < keep.size(); ++c)
    for (int t = 0; t < 3; ++t) {
      const int i = keep[c] - 1 + t;
      if (i >= 0 && i < n) r[3 * c + t] = tap(a, i, (int)c);
    }
  return r;
}

double min_spacing(const std::vector<double> &x) {
  double h = 1e300;
  for (size_t i = 0; i + 1 < x.size(); ++i) h = std::min(h, x[i + 1] - x[i]);
  return h;
}

struct Term {
  int c;
  double w;
};

// Coarse nodes (linear index on the coarse grid) and weights interpolating
// into fine node (i, j, k): up to 8.
int interp_terms(const MgLevel &f, const MgLevel &c, int i, int j, int k, Term *out) {
  const int ci[2] = {f.ax.c0[i], f.ax.c1[i]}, cj[2] = {f.ay.c0[j], f.ay.c1[j]}, ck[2] = {f.az.c0[k], f.az.c1[k]};
  const double wi[2] = {f.ax.w0[i], f.ax.w1[i]}, wj[2] = {f.ay.w0[j], f.ay.w1[j]}, wk[2] = {f.az.w0[k], f.az.w1[k]};
  int n = 0;
  for (int a = 0; a < 2; ++a) {
    if (wi[a] == 0.0) continue;
    for (int b = 0; b < 2; ++b) {
      if (wj[b] == 0.0) continue;
      for (int d = 0; d < 2; ++d) {
        if (wk[d] == 0.0) continue;
        const int C = c.idx(ci[a], cj[b], ck[d]);
        if (c.dir[C]) continue;  // zero on a Dirichlet coarse node
        out[n++] = Term{C, wi[a] * wj[b] * wk[d]};
      }
    }
  }
  return n;
}

// Gauss-Jordan inverse with partial pivoting; a vanishing pivot (a floating
// subsystem) becomes an identity row.
std::vector<double> dense_inverse(std::vector<double> a, int n) {
  std::vector<double> inv((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) inv[(size_t)i * n + i] = 1.0;
  double scale = 0;
  for (double v : a) scale = std::max(scale, std::fabs(v));
  for (int col = 0; col < n; ++col) {
    int piv = col;
    for (int r = col + 1; r < n; ++r)
      if (std::fabs(a[(size_t)r * n + col]) > std::fabs(a[(size_t)piv * n + col])) piv = r;
    if (std::fabs(a[(size_t)piv * n + col]) <= 1e-14 * scale) {
      for (int q = 0; q < n; ++q) { a[(size_t)col * n + q] = 0.0; a[(size_t)q * n + col] = 0.0; }
      a[(size_t)col * n + col] = 1.0;
      piv = col;
    }
    if (piv != col)
      for (int q = 0; q < n; ++q) {
        std::swap(a[(size_t)piv * n + q], a[(size_t)col * n + q]);
        std::swap(inv[(size_t)piv * n + q], inv[(size_t)col * n + q]);
      }
    const double d = 1.0 / a[(size_t)col * n + col];
    for (int q = 0; q < n; ++q) { a[(size_t)col * n + q] *= d; inv[(size_t)col * n + q] *= d; }
    for (int r = 0; r < n; ++r) {
      if (r == col) continue;
      const double f = a[(size_t)r * n + col];
      if (f == 0.0) continue;
      for (int q = 0; q < n; ++q) {
        a[(size_t)r * n + q] -= f * a[(size_t)col * n + q];
        inv[(size_t)r * n + q] -= f * inv[(size_t)col * n + q];
      }
    }
  }
  return inv;
}

// y = A x on the free rows of level l (level 0: the 7-point stencil; decoupled
// rows and neighbours excluded).
void apply_level(const MgLevel &L, const std::vector<double> *st7, const std::vector<double> &x,
                 std::vector<double> &y) {
  for (int j = 0; j < L.py; ++j)
    for (int i = 0; i < L.px; ++i)
      for (int k = 0; k < L.pz; ++k) {
        const int I = L.idx(i, j, k);
        if (L.dir[I]) {
          y[I] = 0.0;
          continue;
        }
        double acc = 0.0;
        if (st7) {
          const double *s = &(*st7)[(size_t)I * 7];
          acc = s[6] * x[I];
          const int nb[6] = {i > 0 ? I - L.pz : -1, i + 1 < L.px ? I + L.pz : -1, j > 0 ? I - L.px * L.pz : -1,
                             j + 1 < L.py ? I + L.px * L.pz : -1, k > 0 ? I - 1 : -1, k + 1 < L.pz ? I + 1 : -1};
          for (int q = 0; q < 6; ++q)
            if (nb[q] >= 0 && !L.dir[nb[q]]) acc += s[q] * x[nb[q]];
        } else {
          for (int di = -1; di <= 1; ++di)
            for (int dj = -1; dj <= 1; ++dj)
              for (int dk = -1; dk <= 1; ++dk) {
                const int i2 = i + di, j2 = j + dj, k2 = k + dk;
                if (i2 < 0 || j2 < 0 || k2 < 0 || i2 >= L.px || j2 >= L.py || k2 >= L.pz) continue;
                acc += L.st[(size_t)I * 27 + ((di + 1) * 3 + (dj + 1)) * 3 + (dk + 1)] * x[L.idx(i2, j2, k2)];
              }
        }
        y[I] = acc;
      }
}

// Largest eigenvalue of D^-1 A on the free rows by power iteration from a
// fixed pseudo-random start (40 steps; it approaches from below, which the
// damping margin covers).
double spectral_radius(const MgLevel &L, const std::vector<double> *st7) {
  const int n = L.nodes();
  std::vector<double> v(n), w(n);
  uint64_t h = 0x9E3779B97F4A7C15ull;
  for (int i = 0; i < n; ++i) {
    h ^= h >> 33; h *= 0xff51afd7ed558ccdull; h ^= h >> 33; h += 0x9E3779B97F4A7C15ull;
    v[i] = L.dir[i] ? 0.0 : (double)(h >> 11) * 0x1p-53 - 0.5;
  }
  double lam = 0.0;
  for (int it = 0; it < 40; ++it) {
    double vv = 0.0;
    for (int i = 0; i < n; ++i) vv += v[i] * v[i];
    if (vv == 0.0) return 1.0;
    apply_level(L, st7, v, w);
    double ww = 0.0;
    for (int i = 0; i < n; ++i) {
      w[i] *= L.dinv[i];
      ww += w[i] * w[i];
    }
    lam = std::sqrt(ww / vv);
    const double inv = 1.0 / std::sqrt(ww > 0 ? ww : 1.0);
    for (int i = 0; i < n; ++i) v[i] = w[i] * inv;
  }
  return lam > 0.0 ? lam : 1.0;
}

}  // namespace

MgHierarchy MgHierarchy::build(int px, int py, int pz, const std::vector<double> &x, const std::vector<double> &y,
                               const std::vector<double> &z, const std::vector<double> &stencil7,
                               const std::vector<uint8_t> &dirichlet) {
  MgHierarchy h;
  {
    MgLevel l0;
    l0.px = px; l0.py = py; l0.pz = pz;
    l0.x = x; l0.y = y; l0.z = z;
    l0.dir.resize(l0.nodes());
    l0.dinv.resize(l0.nodes());
    for (int n = 0; n < l0.nodes(); ++n) {
      const double *a = &stencil7[(size_t)n * 7];
      const bool isolated = a[0] == 0.0 && a[1] == 0.0 && a[2] == 0.0 && a[3] == 0.0 && a[4] == 0.0 && a[5] == 0.0;
      l0.dir[n] = dirichlet[n] || isolated;
      l0.dinv[n] = dirichlet[n] ? 0.0 : 1.0 / a[6];
    }
    h.levels.push_back(std::move(l0));
  }
  for (;;) {
    MgLevel &f = h.levels.back();
    if (f.nodes() <= kMgCoarseMax || (int)h.levels.size() >= kMgMaxLevels) break;
    const double hmin = std::min(min_spacing(f.x), std::min(min_spacing(f.y), min_spacing(f.z)));
    std::vector<int> kx, ky, kz;
    // widen the cut until some interval merges (a graded axis can leave
    // every pair above twice the finest spacing)
    for (double hcut = 2.0 * hmin * (1.0 + 1e-9); hcut < 1e300; hcut *= 2.0) {
      kx = select_axis(f.x, hcut);
      ky = select_axis(f.y, hcut);
      kz = select_axis(f.z, hcut);
      if ((int)(kx.size() * ky.size() * kz.size()) < f.nodes()) break;
      if (kx.size() <= 2 && ky.size() <= 2 && kz.size() <= 2) break;
    }
    if ((int)(kx.size() * ky.size() * kz.size()) == f.nodes()) break;
    MgLevel c;
    c.px = (int)kx.size(); c.py = (int)ky.size(); c.pz = (int)kz.size();
    for (int i : kx) c.x.push_back(f.x[i]);
    for (int j : ky) c.y.push_back(f.y[j]);
    for (int k : kz) c.z.push_back(f.z[k]);
    f.kx = kx;
    f.ky = ky;
    f.kz = kz;
    f.ax = make_axis(f.x, kx);
    f.ay = make_axis(f.y, ky);
    f.az = make_axis(f.z, kz);
    f.rx = restriction_taps(f.ax, kx);
    f.ry = restriction_taps(f.ay, ky);
    f.rz = restriction_taps(f.az, kz);
    // a coarse node on a decoupled fine node is decoupled too: interpolation
    // then falls to zero at Dirichlet walls instead of reaching across them
    c.dir.assign(c.nodes(), 0);
    for (int j = 0; j < c.py; ++j)
      for (int i = 0; i < c.px; ++i)
        for (int k = 0; k < c.pz; ++k) c.dir[c.idx(i, j, k)] = f.dir[f.idx(kx[i], ky[j], kz[k])];
    c.st.assign((size_t)c.nodes() * 27, 0.0);
    const bool fine0 = h.levels.size() == 1;
    Term ti[8], tj[8];
    for (int j = 0; j < f.py; ++j)
      for (int i = 0; i < f.px; ++i)
        for (int k = 0; k < f.pz; ++k) {
          const int I = f.idx(i, j, k);
          if (f.dir[I]) continue;
          const int ni = interp_terms(f, c, i, j, k, ti);
          auto couple = [&](int i2, int j2, int k2, double a) {
            if (a == 0.0 || i2 < 0 || j2 < 0 || k2 < 0 || i2 >= f.px || j2 >= f.py || k2 >= f.pz) return;
            if (f.dir[f.idx(i2, j2, k2)]) return;
            const int nj = interp_terms(f, c, i2, j2, k2, tj);
            for (int a1 = 0; a1 < ni; ++a1) {
              const int C1 = ti[a1].c;
              const int c1k = C1 % c.pz, c1i = (C1 / c.pz) % c.px, c1j = C1 / (c.pz * c.px);
              for (int a2 = 0; a2 < nj; ++a2) {
                const int C2 = tj[a2].c;
                const int c2k = C2 % c.pz, c2i = (C2 / c.pz) % c.px, c2j = C2 / (c.pz * c.px);
                const int di = c2i - c1i, dj = c2j - c1j, dk = c2k - c1k;
                if (di < -1 || di > 1 || dj < -1 || dj > 1 || dk < -1 || dk > 1)
                  throw std::logic_error("multigrid: coarse coupling wider than one node");
                c.st[(size_t)C1 * 27 + ((di + 1) * 3 + (dj + 1)) * 3 + (dk + 1)] += ti[a1].w * a * tj[a2].w;
              }
            }
          };
          if (fine0) {
            const double *s = &stencil7[(size_t)I * 7];
            couple(i - 1, j, k, s[0]);
            couple(i + 1, j, k, s[1]);
            couple(i, j - 1, k, s[2]);
            couple(i, j + 1, k, s[3]);
            couple(i, j, k - 1, s[4]);
            couple(i, j, k + 1, s[5]);
            couple(i, j, k, s[6]);
          } else {
            const double *s = &f.st[(size_t)I * 27];
            for (int di = -1; di <= 1; ++di)
              for (int dj = -1; dj <= 1; ++dj)
                for (int dk = -1; dk <= 1; ++dk)
                  couple(i + di, j + dj, k + dk, s[((di + 1) * 3 + (dj + 1)) * 3 + (dk + 1)]);
          }
        }
    c.dinv.assign(c.nodes(), 0.0);
    for (int n = 0; n < c.nodes(); ++n) {
      const double d = c.st[(size_t)n * 27 + 13];
      if (c.dir[n]) continue;
      if (d > 0.0) c.dinv[n] = 1.0 / d;
      else c.dir[n] = 1;
    }
    h.levels.push_back(std::move(c));
  }
  if (h.levels.back().nodes() > 4 * kMgCoarseMax)
    throw std::runtime_error("multigrid: the mesh does not coarsen to a direct solve");
  // damped-Jacobi weights: omega * rho(D^-1 A) = 1.6
  for (size_t l = 0; l + 1 < h.levels.size(); ++l)
    h.levels[l].omega = 1.6 / spectral_radius(h.levels[l], l == 0 ? &stencil7 : nullptr);
  // exact solve on the coarsest level
  const MgLevel &cl = h.levels.back();
  const int n = cl.nodes();
  std::vector<double> a((size_t)n * n, 0.0);
  if (h.levels.size() == 1) {  // a fine grid small enough to solve directly
    for (int j = 0; j < py; ++j)
      for (int i = 0; i < px; ++i)
        for (int k = 0; k < pz; ++k) {
          const int I = cl.idx(i, j, k);
          const double *s = &stencil7[(size_t)I * 7];
          if (dirichlet[I]) {
            a[(size_t)I * n + I] = 1.0;
            continue;
          }
          a[(size_t)I * n + I] = s[6];
          const int nb[6] = {i > 0 ? I - pz : -1, i + 1 < px ? I + pz : -1, j > 0 ? I - px * pz : -1,
                             j + 1 < py ? I + px * pz : -1, k > 0 ? I - 1 : -1, k + 1 < pz ? I + 1 : -1};
          for (int q = 0; q < 6; ++q)
            if (nb[q] >= 0 && s[q] != 0.0 && !dirichlet[nb[q]]) a[(size_t)I * n + nb[q]] += s[q];
        }
    h.coarse_inv = dense_inverse(std::move(a), n);
    return h;
  }
  for (int j = 0; j < cl.py; ++j)
    for (int i = 0; i < cl.px; ++i)
      for (int k = 0; k < cl.pz; ++k) {
        const int I = cl.idx(i, j, k);
        if (cl.dir[I]) {
          a[(size_t)I * n + I] = 1.0;
          continue;
        }
        for (int di = -1; di <= 1; ++di)
          for (int dj = -1; dj <= 1; ++dj)
            for (int dk = -1; dk <= 1; ++dk) {
              const int i2 = i + di, j2 = j + dj, k2 = k + dk;
              if (i2 < 0 || j2 < 0 || k2 < 0 || i2 >= cl.px || j2 >= cl.py || k2 >= cl.pz) continue;
              const int J = cl.idx(i2, j2, k2);
              if (cl.dir[J]) continue;
              a[(size_t)I * n + J] += cl.st[(size_t)I * 27 + ((di + 1) * 3 + (dj + 1)) * 3 + (dk + 1)];
            }
      }
  h.coarse_inv = dense_inverse(std::move(a), n);
  return h;
}

}  // namespace mcb200
