// mg_kernels.h -- the multigrid-preconditioned CG Poisson solve on the GPU
// (mg_kernels.cu): device copy of an MgHierarchy and its launcher.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "mg_setup.h"

namespace mcb200 {

struct MgDevLevel {
  int px = 0, py = 0, pz = 0, n = 0;
  double omega = 0.0;
  const double *st = nullptr;    // stencil, coefficient-major: [7][n] the CG's (level 0), [27][n] Galerkin
  const double *dinv = nullptr;  // [n] 1 / diagonal, 0 on Dirichlet rows
  const uint8_t *dir = nullptr;  // [n] decoupled rows
  double *b = nullptr, *xa = nullptr, *xb = nullptr, *r = nullptr;  // right side, iterate (ping-pong), residual
  // interpolation from the next coarser level into this one, per axis:
  // (c0, c1) coarse indices and (w0, w1) weights of each fine index, and the
  // fine index of each coarse node
  const int2 *cmap[3] = {nullptr, nullptr, nullptr};
  const double2 *wmap[3] = {nullptr, nullptr, nullptr};
  const int *keep[3] = {nullptr, nullptr, nullptr};
  const double *rtap[3] = {nullptr, nullptr, nullptr};  // [3 * coarse] restriction taps (mg_setup.h)
  // level 0 only: [n] the first sweep's factor, x = fscale b (dinv on
  // decoupled rows, omega dinv elsewhere: the same product as the sweep's)
  const double *fscale = nullptr;
};

struct MgDevice {
  int levels = 0;
  int nu = 1;                          // smoothing sweeps before and after the coarse correction
  const double *coarse_inv = nullptr;  // [n][n] dense inverse of the coarsest operator
  MgDevLevel L[kMgMaxLevels];
};

// Copies the hierarchy to the device, with stencil7 ([nodes][7], the CG's)
// as level 0's stencil; every stencil goes coefficient-major.  Level 0's b
// and xa are left null: the solve binds them to the CG residual and
// preconditioned residual.  Every
// allocation is appended to `owned` (freed by the caller with cudaFree).
MgDevice mg_upload(const MgHierarchy &h, const std::vector<double> &stencil7, std::vector<void *> &owned);

// One solve with the V-cycle as preconditioner, in one cooperative launch
// of `grid` blocks: the set-up (the Dirichlet values into x, the initial
// residual and the norms), every CG iteration, the true residual of the
// final iterate and the solve statistics.  Returns the cudaError_t of the
// launch.
struct MgSystem;
cudaError_t launch_cg_mg(const MgSystem &y, int grid, cudaStream_t s);
// Largest cooperative grid of the MG kernel on the current device (blocks per SM x SMs); 0 if unavailable.
int cg_mg_max_grid();
// The MG kernel's default grid, per SM (MCB200_MG_BLOCKS_PER_SM).
int cg_mg_blocks_per_sm();

// One solve's arguments, as launch_cg_mg takes them (mg with level 0's b and
// xa bound to r and z).
struct MgSystem {
  MgDevice mg;
  const double *st7 = nullptr;
  const uint8_t *dirichlet = nullptr;
  // r and r1: the CG residual, alternating each iteration
  double *x = nullptr, *r = nullptr, *r1 = nullptr, *p0 = nullptr, *p1 = nullptr, *q = nullptr, *part = nullptr,
         *sc = nullptr;
  const double *rhs = nullptr;  // right side (Dirichlet rows: the contact values)
  double *stats = nullptr;      // [3] solves, iterations, largest relative residual (accumulated)
  double rel_tol2 = 0.0;        // converged when ||r||^2 <= rel_tol2 ||b_ff||^2
  int px = 0, py = 0, pz = 0, max_iter = 0;
};
// Two solves in one cooperative launch of 2 x `grid` blocks: blocks [0, grid)
// solve a[0], the others a[1], each exactly as launch_cg_mg on `grid` blocks
// (the same node-to-thread mapping and reduction order, so bit-identical
// results), sharing one grid barrier per pass.  Both hierarchies must have
// the same depth and smoothing (the pass sequence); cg_mg_pair_fits says
// whether 2 x grid blocks are co-resident.
cudaError_t launch_cg_mg_pair(const MgSystem a[2], int grid, cudaStream_t s);
bool cg_mg_pair_fits(int grid);

}  // namespace mcb200
