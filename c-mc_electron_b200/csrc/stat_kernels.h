// stat_kernels.h -- window statistics of the particle store (stat_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "device_state.cuh"

namespace mcb200 {

// Fixed-point units of one statistics window, per carrier type (0
// electrons, 1 holes): |q| sums, |q| v sums, |q| E sums.
struct StatScales {
  double q[2], v[2], e[2];
};

struct StatBuffers {
  long long *node = nullptr;                 // [2 types][5: qvx qvy qvz q qE][nodes]
  unsigned long long *cell_count = nullptr;  // [cells]
  double *pot_sum = nullptr;                 // [nodes]
  double *qc_pot_sum = nullptr;              // [nodes] the electrons' potential (quantum-corrected when on)
  int nodes = 0;
};

template <typename R>
void launch_statistic(const DevParticlesT<R> &P, DevCount n, const DevMesh &M, const DevTables &T, const StatScales &S,
                      const StatBuffers &B, int grid, cudaStream_t s);
void launch_add_potential(int nodes, const double *pot, double *sum, cudaStream_t s);

// Induced (Ramo-Shockley) current of one contact over the store: the sum
// over live particles of q v . E_w (v the group velocity, E_w[cells][3] the
// contact's weighting field) added to sum[0], and 1 to sum[1] (steps).  The
// particle terms are summed in int64 fixed point (acc) with a unit from the
// store's charge bounds (bounds[4], the context's, kept current by every
// writer of the store), so the result does not
// depend on the store's order; the step's total is then added to the FP64
// running sum by one thread.  vmax, emax: bounds on |v| and |E_w| components.
struct InducedBuffers {
  const double *field = nullptr;
  const unsigned long long *bounds = nullptr;  // [4] charge bounds of the store
  long long *acc = nullptr;              // [1]
  double *sum = nullptr;                 // [2]
  double vmax = 0, emax = 0;
};
template <typename R>
void launch_induced_current(const DevParticlesT<R> &P, DevCount n, const DevMesh &M, const DevTables &T,
                            const InducedBuffers &B, int grid, cudaStream_t s);

}  // namespace mcb200
