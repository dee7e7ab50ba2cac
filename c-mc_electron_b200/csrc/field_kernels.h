// field_kernels.h -- device buffers and launchers of deposition, the Poisson
// solve and the field update (field_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "device_state.cuh"
#include "mg_kernels.h"

namespace mcb200 {

// Fixed-point units (powers of two) of the deposition sums: electron cell
// charge, hole cell charge, |charge| and node charge.
struct DepositScales {
  double s[3];
};

struct FieldBuffers {
  // device description (poisson_setup.h), uploaded once
  double *cvol = nullptr, *pvol = nullptr, *pdop = nullptr, *vadd = nullptr;
  double *stencil = nullptr, *diag_inv = nullptr;
  uint8_t *dirichlet = nullptr;
  double *bc_vapp = nullptr, *bc_phims = nullptr;
  // deposition results
  long long *acc_cell = nullptr;  // [3][cells] fixed-point sums: electron q, hole q, |q|
  long long *acc_node = nullptr;  // [nodes]
  double *cell_e = nullptr, *cell_h = nullptr;  // c_electron_charge, c_hole_charge
  double *density = nullptr;                    // p_par_charge (charge / node volume)
  // Poisson
  double *rhs = nullptr, *potential = nullptr;
  double *cg_r = nullptr, *cg_r1 = nullptr, *cg_z = nullptr, *cg_p = nullptr, *cg_p1 = nullptr, *cg_q = nullptr, *cg_part = nullptr,
         *cg_scalars = nullptr;
  unsigned long long *abs_sum = nullptr;  // [4] charge bounds of the store (the context's, kept by its writers)
  const MgDevice *mg = nullptr;  // multigrid hierarchy of the stencil (null: Jacobi preconditioning only)
  double *poisson_stats = nullptr;  // [3] solves, iterations, largest relative residual (since the last reset)
};

// out[4] = {max |q| bits of electrons, of holes, electron count, hole count}
template <typename R>
void launch_charge_bounds(const DevParticlesT<R> &P, DevCount n, unsigned long long *out, int grid, cudaStream_t s);
// The deposition sums, with fixed-point units from the store's charge
// bounds (f.abs_sum, current when the deposition starts), all on the
// device: nothing waits for the host.  f.acc_cell and f.acc_node must hold
// zeros on entry and do again on exit.
template <typename R>
void launch_deposit(const DevParticlesT<R> &P, DevCount n, const DevMesh &M, const FieldBuffers &f, int grid,
                    cudaStream_t s);
void launch_rhs(int nodes, const FieldBuffers &f, cudaStream_t s);
// The CG iterations of one solve run in one cooperative launch; its grid
// (blocks) is fixed per context on first use, so the reduction order is too.
constexpr int kCgMaxGrid = 1024;
enum CgMethod { kCgAuto = 0, kCgJacobi = 1, kCgMultigrid = 2 };
struct CgPlan {
  int method = kCgAuto;  // kCgAuto: multigrid when the hierarchy exists
  int blocks = 0;        // requested grid (0: Jacobi the largest co-resident grid up to kCgMaxGrid, multigrid 1 per SM)
  int grid = 0;          // grid in use (0 until the first solve)
  int used = 0;          // kCgJacobi or kCgMultigrid, set by the last solve
  double rel_tol2 = 0;   // the last cg_prepare's rel_tol^2
  unsigned long long launches = 0;
};
// Returns 0 on success; host_scratch must hold 10 doubles (pinned).  With
// iterations and rel_residual both null nothing waits for the GPU (the
// results only reach f.poisson_stats).
int cg_solve(const DevMesh &M, const FieldBuffers &f, double rel_tol, int max_iter, cudaStream_t s,
             double *host_scratch, int *iterations, double *rel_residual, CgPlan &plan);
// cg_solve in three parts, for callers that launch several solves together:
// the set-up (Jacobi: residual and tolerances; both: the plan's grid and
// tolerance), the persistent launch (multigrid: set-up, iterations, true
// residual and statistics in one), then (Jacobi) the true residual and
// statistics and (both) the results to the host when asked for.  Each
// returns 0 on success.  cg_mg_system: the multigrid launch's arguments
// (plan.used == kCgMultigrid, after cg_prepare) for launch_cg_mg_pair.
int cg_prepare(const DevMesh &M, const FieldBuffers &f, double rel_tol, cudaStream_t s, CgPlan &plan);
int cg_launch(const DevMesh &M, const FieldBuffers &f, int max_iter, cudaStream_t s, CgPlan &plan);
int cg_finish(const DevMesh &M, const FieldBuffers &f, const CgPlan &plan, cudaStream_t s, double *host_scratch,
              int *iterations, double *rel_residual);
MgSystem cg_mg_system(const DevMesh &M, const FieldBuffers &f, int max_iter, double rel_tol2);
// Fields of both carriers from pot; with pot_e, the electrons' from pot_e.
void launch_pot2field(const DevMesh &M, const double *pot, cudaStream_t s, const double *pot_e = nullptr);

}  // namespace mcb200
