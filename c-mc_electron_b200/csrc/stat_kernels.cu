// stat_kernels.cu -- the per-step statistics the reference writes every
// stat_step steps (MeshQuantities::statistic, src/mcmodel.cpp:1167-1408):
// per node and carrier type the CIC-weighted |q| v_x, |q| v_y, |q| v_z,
// |q| and |q| E of every particle, per cell the particle count, and per node
// the potential; summed over the steps of a statistics window.
//
// Node sums are int64 fixed point (order independent).  A window's scales
// are fixed when it starts, from bounds every sum respects for the whole
// window: |q| sums <= (particles of the type) x max|q| x steps x 4 (the
// factor leaves room for GENERATE copies and refreshes), |v| <= the
// largest group-velocity component of the band tables, |E| <= the energy
// table's top.
#include "stat_kernels.h"

namespace mcb200 {

constexpr uint32_t kStatDead = 1u << 16;

__device__ __forceinline__ void st_add(long long *p, double v, double scale) {
  atomicAdd(reinterpret_cast<unsigned long long *>(p), (unsigned long long)__double2ll_rn(v * scale));
}

// GetV (src/ParticleUtils.cpp:307-313) from the FP64 tables: the wedge
// velocity of itet mapped out of the wedge of isym.
__device__ __forceinline__ void group_velocity(const DevTables &T, int itet, int isym, double &vx, double &vy,
                                               double &vz) {
  const double *v = T.tf[itet].v;
  const int *m = T.symi + isym * 6;  // matsym[c][isym] at isym * 6 + c
  const int p0 = m[0] - 1, p1 = m[1] - 1, p2 = m[2] - 1;
  vx = (p0 == 0 ? v[0] : (p0 == 1 ? v[1] : v[2])) * (double)m[3];
  vy = (p1 == 0 ? v[0] : (p1 == 1 ? v[1] : v[2])) * (double)m[4];
  vz = (p2 == 0 ? v[0] : (p2 == 1 ? v[1] : v[2])) * (double)m[5];
}

template <typename R>
__global__ void statistic_kernel(DevParticlesT<R> P, DevCount count, DevMesh M, DevTables T, StatScales S,
                                 StatBuffers B) {
  const int n = count.get();
  const int px = M.nx + 1, pz = M.nz + 1;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const uint32_t meta = P.meta[p];
    if (meta & kStatDead) continue;
    const uint32_t c = P.cell[p];
    const int i = c & 1023, j = (c >> 10) & 1023, k = (c >> 20) & 1023;
    atomicAdd(B.cell_count + (j * M.nx + i) * M.nz + k, 1ull);
    const int type = ((meta >> 8) & 255) == 0 ? 0 : 1;
    double vx, vy, vz;
    group_velocity(T, P.itet[p], meta & 255, vx, vy, vz);
    double rx, ry, rz;
    if constexpr (sizeof(R) == 4) {
      rx = (double)P.x[p] / M.dx[i];
      ry = (double)P.y[p] / M.dy[j];
      rz = (double)P.z[p] / M.dz[k];
    } else {
      rx = (P.x[p] - M.lx[i]) / M.dx[i];
      ry = (P.y[p] - M.ly[j]) / M.dy[j];
      rz = (P.z[p] - M.lz[k]) / M.dz[k];
    }
    const double q = P.charge[p], e = P.energy[p];
    long long *base = B.node + (size_t)type * 5 * B.nodes;
    const double sq = S.q[type], sv = S.v[type], se = S.e[type];
    auto put = [&](int a, int b, int d, double w) {
      const size_t node = ((size_t)b * px + a) * pz + d;
      const double aq = fabs(q * w);
      st_add(base + 0 * (size_t)B.nodes + node, vx * aq, sv);
      st_add(base + 1 * (size_t)B.nodes + node, vy * aq, sv);
      st_add(base + 2 * (size_t)B.nodes + node, vz * aq, sv);
      st_add(base + 3 * (size_t)B.nodes + node, aq, sq);
      st_add(base + 4 * (size_t)B.nodes + node, aq * e, se);
    };
    // the eight corners in the reference's order and weights
    put(i, j, k, (1 - rx) * (1 - ry) * (1 - rz));
    put(i + 1, j, k, rx * (1 - ry) * (1 - rz));
    put(i, j, k + 1, (1 - rx) * (1 - ry) * rz);
    put(i + 1, j, k + 1, rx * (1 - ry) * rz);
    put(i, j + 1, k, (1 - rx) * ry * (1 - rz));
    put(i + 1, j + 1, k, rx * ry * (1 - rz));
    put(i, j + 1, k + 1, (1 - rx) * ry * rz);
    put(i + 1, j + 1, k + 1, rx * ry * rz);
  }
}

// stat_pot += pot: one thread per node, so the FP64 sum is exact to the
// reference's order (step by step).
__global__ void add_potential_kernel(int nodes, const double *pot, double *sum) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < nodes) sum[p] += pot[p];
}

template <typename R>
void launch_statistic(const DevParticlesT<R> &P, DevCount n, const DevMesh &M, const DevTables &T, const StatScales &S,
                      const StatBuffers &B, int grid, cudaStream_t s) {
  statistic_kernel<R><<<grid, 256, 0, s>>>(P, n, M, T, S, B);
}
void launch_add_potential(int nodes, const double *pot, double *sum, cudaStream_t s) {
  if (nodes > 0 && pot) add_potential_kernel<<<(nodes + 255) / 256, 256, 0, s>>>(nodes, pot, sum);
}

template void launch_statistic<double>(const DevParticlesT<double> &, DevCount, const DevMesh &, const DevTables &,
                                       const StatScales &, const StatBuffers &, int, cudaStream_t);
template void launch_statistic<float>(const DevParticlesT<float> &, DevCount, const DevMesh &, const DevTables &,
                                      const StatScales &, const StatBuffers &, int, cudaStream_t);

}  // namespace mcb200
