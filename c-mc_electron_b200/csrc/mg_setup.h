// mg_setup.h -- geometric multigrid hierarchy for the Poisson CG
// preconditioner, built on the host once per device description.
//
// Levels are vertex grids.  Per axis the first and last node are kept and
// an interior node is dropped where the interval it splits is no wider than
// twice the level's finest spacing (never two consecutive nodes), so finely
// spaced regions coarsen first: on a graded mesh anisotropic cells coarsen
// along their short sides only.  Interpolation is linear along each axis in
// the node coordinates, trilinear in 3-D, with the rows of decoupled
// (Dirichlet) fine nodes zeroed.  Coarse operators are Galerkin products
// P^T A P: the fine level is the 7-point finite-volume stencil of the free
// nodes, every coarse level a 27-point stencil.  Coarsening stops at
// kMgCoarseMax nodes, where the V-cycle solves exactly with a dense inverse.
#pragma once

#include <cstdint>
#include <vector>

namespace mcb200 {

constexpr int kMgCoarseMax = 512;
constexpr int kMgMaxLevels = 10;

struct MgAxis {              // interpolation of one axis: fine index -> two coarse nodes
  std::vector<int> c0, c1;   // coarse indices (c1 == c0 with w1 = 0 at coarse nodes)
  std::vector<double> w0, w1;
};

struct MgLevel {
  int px = 0, py = 0, pz = 0;      // nodes per axis
  double omega = 0.0;              // damped-Jacobi weight of the smoother (not used on the coarsest level)
  std::vector<double> st;          // level 0: empty (the 7-point stencil is the CG's); else 27 per node
  std::vector<double> dinv;        // 1 / diagonal; 0 on Dirichlet rows
  std::vector<uint8_t> dir;        // decoupled rows: Dirichlet, or (level 0) isolated nodes without
                                   // neighbours (all-vacuum corners), which the V-cycle solves by dinv alone
  std::vector<double> x, y, z;     // node coordinates
  MgAxis ax, ay, az;               // interpolation from level + 1 into this level (empty on the coarsest)
  std::vector<int> kx, ky, kz;     // fine index of each node of level + 1, per axis (empty on the coarsest)
  // restriction taps per axis: for node c of level + 1, the weights of the
  // fine indices kx[c] - 1, kx[c], kx[c] + 1 (0 off the grid) -- [3 * coarse]
  std::vector<double> rx, ry, rz;
  int nodes() const { return px * py * pz; }
  int idx(int i, int j, int k) const { return (j * px + i) * pz + k; }
};

struct MgHierarchy {
  std::vector<MgLevel> levels;
  std::vector<double> coarse_inv;  // dense inverse of the coarsest operator [n][n]

  // stencil7: [nodes][7] (-x, +x, -y, +y, -z, +z, diagonal) of the node grid
  // px x py x pz, node (i, j, k) at (j * px + i) * pz + k; dirichlet per node.
  static MgHierarchy build(int px, int py, int pz, const std::vector<double> &x, const std::vector<double> &y,
                           const std::vector<double> &z, const std::vector<double> &stencil7,
                           const std::vector<uint8_t> &dirichlet);
};

}  // namespace mcb200
