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

}  // namespace mcb200
