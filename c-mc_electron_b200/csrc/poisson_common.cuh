// poisson_common.cuh -- helpers shared by the Poisson kernels: node
// indexing of the vertex grid and fixed-order block reductions.
#pragma once

#include <cuda_runtime.h>

namespace mcb200 {

// node (i, j, k) of a px x py x pz vertex grid is (j * px + i) * pz + k
struct Grid3 {
  int px, py, pz;
};
__device__ __forceinline__ void node_ijk(int p, const Grid3 &g, int &i, int &j, int &k) {
  k = p % g.pz;
  const int t = p / g.pz;
  i = t % g.px;
  j = t / g.px;
}

constexpr int kRedBlock = 256;

// Fixed-order block partial sums of a[i]*b[i] (first stage of a dot product).
template <int B>
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double s[B];
  s[threadIdx.x] = v;
  __syncthreads();
  for (int o = B / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
    __syncthreads();
  }
  const double r = s[0];
  __syncthreads();
  return r;
}

// Sum of n partials, read in the same order by every block.
__device__ __forceinline__ double sum_partials(const double *part, int n) {
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += kRedBlock) v += part[i];
  return block_sum<kRedBlock>(v);
}

}  // namespace mcb200
