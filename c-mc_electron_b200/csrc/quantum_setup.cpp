// quantum_setup.cpp -- host set-up of the effective-potential quantum
// correction (quantum_setup.h).
#include "quantum_setup.h"

#include <algorithm>
#include <stdexcept>

namespace mcb200 {

namespace {

constexpr int kOxide = 2, kSilicon = 3;  // material tokens (include/Constant_GlobalVariable_MathFunction.h:167-169)
constexpr double kSqrt2 = 1.4142135623730950488e0;

// Node flags as init_p_mat sets them (include/defs.h:129-137).
enum : unsigned {
  kNodeSilicon = 1u,
  kNodeOxide = 2u,
  kNodeUp = 1u << 2,
  kNodeDown = 1u << 3,
  kNodeFront = 1u << 4,
  kNodeBack = 1u << 5,
  kNodeLeft = 1u << 6,
  kNodeRight = 1u << 7,
  kNodeQuantum = 1u << 8,
};

// The window [lower, upper] of every node index along one axis, as
// init_effective_potential finds it (src/mcmodel.cpp:2589-2630): the node
// before the first coordinate >= x - w (searching up to the node itself),
// and the first coordinate > x + w (the last node when there is none).  The
// search iterators carry over from one node to the next, as there.
void axis_window(const std::vector<double> &l, double w, int *lower, int *upper) {
  auto low = l.begin(), up = l.begin();
  for (size_t i = 0; i < l.size(); ++i) {
    low = std::lower_bound(low, l.begin() + i, l[i] - w);
    up = std::upper_bound(up, l.end(), l[i] + w);
    if (low != l.begin()) --low;
    if (up == l.end()) --up;
    lower[i] = (int)(low - l.begin());
    upper[i] = (int)(up - l.begin());
  }
}

}  // namespace

QuantumHost quantum_setup(int nx, int ny, int nz, const double *lx, const double *ly, const double *lz,
                          const double *dx, const double *dy, const double *dz, const int32_t *material,
                          const int32_t *quantum_region, const QuantumParams &p) {
  for (int a = 0; a < 3; ++a)
    if (!(p.theta[a] > 0)) throw std::invalid_argument("quantum correction: theta must be positive on every axis");
  const int px = nx + 1, py = ny + 1, pz = nz + 1;
  const size_t nodes = (size_t)px * py * pz;
  auto node = [&](int i, int j, int k) { return ((size_t)j * px + i) * pz + k; };
  // init_p_mat (src/mcmodel.cpp:2495-2582): every corner of a quantum /
  // silicon / oxide cell carries the flag
  std::vector<unsigned> mat(nodes, 0u);
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i)
      for (int k = 0; k < nz; ++k) {
        const size_t c = ((size_t)j * nx + i) * nz + k;
        unsigned f = 0;
        if (quantum_region && quantum_region[c]) f |= kNodeQuantum;
        if (material[c] == kSilicon) f |= kNodeSilicon;
        if (material[c] == kOxide) f |= kNodeOxide;
        if (!f) continue;
        for (int dj = 0; dj < 2; ++dj)
          for (int di = 0; di < 2; ++di)
            for (int dk = 0; dk < 2; ++dk) mat[node(i + di, j + dj, k + dk)] |= f;
      }
  auto in = [&](int i, int j, int k) { return (mat[node(i, j, k)] & (kNodeOxide | kNodeSilicon)) != 0; };
  std::vector<unsigned> bc(nodes, 0u);
  for (int i = 0; i < px; ++i)
    for (int j = 0; j < py; ++j)
      for (int k = 0; k < pz; ++k) {
        unsigned f = 0;
        if (i == 0 || !in(i - 1, j, k)) f |= kNodeUp;
        if (i == px - 1 || !in(i + 1, j, k)) f |= kNodeDown;
        if (k == 0 || !in(i, j, k - 1)) f |= kNodeFront;
        if (k == pz - 1 || !in(i, j, k + 1)) f |= kNodeBack;
        if (j == 0 || !in(i, j - 1, k)) f |= kNodeLeft;
        if (j == py - 1 || !in(i, j + 1, k)) f |= kNodeRight;
        bc[node(i, j, k)] = f;
      }
  QuantumHost q;
  q.inside.assign(nodes, 0);
  q.eb.assign(nodes, 0.0);
  q.range.assign(6 * nodes, 0.0);
  // init_ep_range (src/mcmodel.cpp:2406-2492)
  const double sx = kSqrt2 * p.theta[0], sy = kSqrt2 * p.theta[1], sz = kSqrt2 * p.theta[2];
  for (int j = 0; j < py; ++j)
    for (int i = 0; i < px; ++i)
      for (int k = 0; k < pz; ++k) {
        const size_t n = node(i, j, k);
        const unsigned m = mat[n], b = bc[n];
        q.inside[n] = (m & (kNodeOxide | kNodeSilicon)) ? 1 : 0;
        if ((m & kNodeOxide) && !(m & kNodeSilicon)) q.eb[n] = -p.eb;
        const double x11 = (b & kNodeUp) ? lx[i] - p.ratio[0] * p.theta[0] : lx[i] - 0.5 * dx[i - 1];
        const double x22 = (b & kNodeDown) ? lx[i] + p.ratio[0] * p.theta[0] : lx[i] + 0.5 * dx[i];
        const double y11 = (b & kNodeLeft) ? ly[j] - p.ratio[1] * p.theta[1] : ly[j] - 0.5 * dy[j - 1];
        const double y22 = (b & kNodeRight) ? ly[j] + p.ratio[1] * p.theta[1] : ly[j] + 0.5 * dy[j];
        const double z11 = (b & kNodeFront) ? lz[k] - p.ratio[2] * p.theta[2] : lz[k] - 0.5 * dz[k - 1];
        const double z22 = (b & kNodeBack) ? lz[k] + p.ratio[2] * p.theta[2] : lz[k] + 0.5 * dz[k];
        q.range[0 * nodes + n] = x11 / sx;
        q.range[1 * nodes + n] = x22 / sx;
        q.range[2 * nodes + n] = y11 / sy;
        q.range[3 * nodes + n] = y22 / sy;
        q.range[4 * nodes + n] = z11 / sz;
        q.range[5 * nodes + n] = z22 / sz;
        if (m & kNodeQuantum) q.list.push_back((int)n);
      }
  // init_effective_potential (src/mcmodel.cpp:2584-2630) and the scaled
  // node coordinates (:2483-2492)
  q.qcl.resize(px + py + pz);
  q.lower.resize(px + py + pz);
  q.upper.resize(px + py + pz);
  const std::vector<double> vx(lx, lx + px), vy(ly, ly + py), vz(lz, lz + pz);
  axis_window(vx, p.ratio[0] * p.theta[0], &q.lower[0], &q.upper[0]);
  axis_window(vy, p.ratio[1] * p.theta[1], &q.lower[px], &q.upper[px]);
  axis_window(vz, p.ratio[2] * p.theta[2], &q.lower[px + py], &q.upper[px + py]);
  for (int i = 0; i < px; ++i) q.qcl[i] = lx[i] / sx;
  for (int j = 0; j < py; ++j) q.qcl[px + j] = ly[j] / sy;
  for (int k = 0; k < pz; ++k) q.qcl[px + py + k] = lz[k] / sz;
  return q;
}

}  // namespace mcb200
