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

// Sum of v over a block of B threads (a multiple of 32), the same bits in
// every thread and on every call: a butterfly within each warp, then every
// thread adds the warp sums in warp order.
template <int B>
__device__ __forceinline__ double block_sum(double v) {
  static_assert(B % 32 == 0 && B <= 1024, "block_sum: whole warps");
  __shared__ double s[B / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = v;
  __syncthreads();
  double r = s[0];
#pragma unroll
  for (int w = 1; w < B / 32; ++w) r += s[w];
  __syncthreads();
  return r;
}

// Sum of n partials, read in the same order by every block of B threads.
template <int B = kRedBlock>
__device__ __forceinline__ double sum_partials(const double *part, int n) {
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += B) v += part[i];
  return block_sum<B>(v);
}

}  // namespace mcb200
