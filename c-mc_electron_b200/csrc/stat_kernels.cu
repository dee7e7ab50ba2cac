// stat_kernels.cu -- the per-step statistics the reference writes every
// stat_step steps (MeshQuantities::statistic, src/mcmodel.cpp:1167-1408):
// per node and carrier type the CIC-weighted |q| v_x, |q| v_y, |q| v_z,
// |q| and |q| E of every particle, per cell the particle count, and per node
// the potential; summed over the steps of a statistics window.  Also the
// current one contact carries by induction (Ramo-Shockley, a tally of the
// transport step): sum over particles of q v . E_w.
//
// Node sums are int64 fixed point (order independent).  A window's scales
// are fixed when it starts, from bounds every sum respects for the whole
// window: |q| sums <= (particles of the type) x max|q| x steps x 4 (the
// factor leaves room for GENERATE copies and refreshes), |v| <= the
// largest group-velocity component of the band tables, |E| <= the energy
// table's top.
#include "stat_kernels.h"
#include "field_kernels.h"
#include "warp_segments.cuh"

namespace mcb200 {

constexpr uint32_t kStatDead = 1u << 16;

__device__ __forceinline__ long long st_fx(double v, double scale) { return __double2ll_rn(v * scale); }
__device__ __forceinline__ void st_put(long long *p, long long v) {
  atomicAdd(reinterpret_cast<unsigned long long *>(p), (unsigned long long)v);
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

// Lanes of a warp walk consecutive particles of the cell-sorted store; runs
// of particles of the same cell and carrier type add their fixed-point
// terms with shuffles before one atomic per run (warp_segments.cuh).
template <typename R>
__global__ void __launch_bounds__(256) statistic_kernel(DevParticlesT<R> P, DevCount count, DevMesh M, DevTables T,
                                                        StatScales S, StatBuffers B) {
  const int n = count.get();
  const int px = M.nx + 1, pz = M.nz + 1;
  const unsigned lane = threadIdx.x & 31u;
  for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += gridDim.x * blockDim.x) {
    const int p = base + (int)lane;
    const uint32_t meta = p < n ? P.meta[p] : kStatDead;
    const bool live = !(meta & kStatDead);
    const uint32_t c = live ? P.cell[p] : 0u;
    const int type = ((meta >> 8) & 255) == 0 ? 0 : 1;
    const WarpRuns runs(live ? (c | ((unsigned)type << 30)) : 0xffffffffu);
    const int i = c & 1023, j = (c >> 10) & 1023, k = (c >> 20) & 1023;
    double vx = 0, vy = 0, vz = 0, rx = 0, ry = 0, rz = 0, q = 0, e = 0;
    if (live) {
      group_velocity(T, P.itet[p], meta & 255, vx, vy, vz);
      if constexpr (sizeof(R) == 4) {
        rx = (double)P.x[p] / M.dx[i];
        ry = (double)P.y[p] / M.dy[j];
        rz = (double)P.z[p] / M.dz[k];
      } else {
        rx = (P.x[p] - M.lx[i]) / M.dx[i];
        ry = (P.y[p] - M.ly[j]) / M.dy[j];
        rz = (P.z[p] - M.lz[k]) / M.dz[k];
      }
      q = P.charge[p];
      e = P.energy[p];
    }
    const long long cnt = runs.sum(live ? 1 : 0);
    if (live && runs.tail)
      atomicAdd(B.cell_count + (j * M.nx + i) * M.nz + k, (unsigned long long)cnt);
    long long *basep = B.node + (size_t)type * 5 * B.nodes;
    const double sq = type ? S.q[1] : S.q[0], sv = type ? S.v[1] : S.v[0], se = type ? S.e[1] : S.e[0];
    auto put = [&](int a, int b, int d, double w) {
      const double aq = fabs(q * w);
      const long long t0 = runs.sum(live ? st_fx(vx * aq, sv) : 0);
      const long long t1 = runs.sum(live ? st_fx(vy * aq, sv) : 0);
      const long long t2 = runs.sum(live ? st_fx(vz * aq, sv) : 0);
      const long long t3 = runs.sum(live ? st_fx(aq, sq) : 0);
      const long long t4 = runs.sum(live ? st_fx(aq * e, se) : 0);
      if (live && runs.tail) {
        const size_t node = ((size_t)b * px + a) * pz + d;
        st_put(basep + 0 * (size_t)B.nodes + node, t0);
        st_put(basep + 1 * (size_t)B.nodes + node, t1);
        st_put(basep + 2 * (size_t)B.nodes + node, t2);
        st_put(basep + 3 * (size_t)B.nodes + node, t3);
        st_put(basep + 4 * (size_t)B.nodes + node, t4);
      }
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

// The fixed-point unit of one step's induced-current terms: sum |q v . E_w|
// <= (electrons + holes) * max|q| * sqrt(3) vmax * sqrt(3) emax.
__device__ __forceinline__ double induced_unit(const unsigned long long *b, double vmax, double emax) {
  const double qmax = fmax(__longlong_as_double((long long)b[0]), __longlong_as_double((long long)b[1]));
  const double bound = fmax((double)(b[2] + b[3]) * qmax * vmax * emax * 3.0, 1e-300);
  return ldexp(1.0, 62 - (int)ceil(log2(bound)));
}

template <typename R>
__global__ void __launch_bounds__(256) induced_current_kernel(DevParticlesT<R> P, DevCount count, DevMesh M,
                                                              DevTables T, InducedBuffers B) {
  const int n = count.get();
  const double unit = induced_unit(B.bounds, B.vmax, B.emax);
  long long t = 0;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const uint32_t meta = P.meta[p];
    if (meta & kStatDead) continue;
    const uint32_t c = P.cell[p];
    const int i = c & 1023, j = (c >> 10) & 1023, k = (c >> 20) & 1023;
    double vx, vy, vz;
    group_velocity(T, P.itet[p], meta & 255, vx, vy, vz);
    const double *ew = B.field + 3 * (size_t)((j * M.nx + i) * M.nz + k);
    t += st_fx(P.charge[p] * (vx * ew[0] + vy * ew[1] + vz * ew[2]), unit);
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) t += __shfl_down_sync(0xffffffffu, t, off);
  if ((threadIdx.x & 31u) == 0 && t) st_put(B.acc, t);
}
__global__ void induced_finish_kernel(InducedBuffers B) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    B.sum[0] += (double)*B.acc / induced_unit(B.bounds, B.vmax, B.emax);
    B.sum[1] += 1.0;
    *B.acc = 0;
  }
}

template <typename R>
void launch_statistic(const DevParticlesT<R> &P, DevCount n, const DevMesh &M, const DevTables &T, const StatScales &S,
                      const StatBuffers &B, int grid, cudaStream_t s) {
  statistic_kernel<R><<<grid, 256, 0, s>>>(P, n, M, T, S, B);
}
void launch_add_potential(int nodes, const double *pot, double *sum, cudaStream_t s) {
  if (nodes > 0 && pot) add_potential_kernel<<<(nodes + 255) / 256, 256, 0, s>>>(nodes, pot, sum);
}

template <typename R>
void launch_induced_current(const DevParticlesT<R> &P, DevCount n, const DevMesh &M, const DevTables &T,
                            const InducedBuffers &B, int grid, cudaStream_t s) {
  induced_current_kernel<R><<<grid, 256, 0, s>>>(P, n, M, T, B);
  induced_finish_kernel<<<1, 32, 0, s>>>(B);
}
template void launch_induced_current<double>(const DevParticlesT<double> &, DevCount, const DevMesh &,
                                             const DevTables &, const InducedBuffers &, int, cudaStream_t);
template void launch_induced_current<float>(const DevParticlesT<float> &, DevCount, const DevMesh &,
                                            const DevTables &, const InducedBuffers &, int, cudaStream_t);
template void launch_statistic<double>(const DevParticlesT<double> &, DevCount, const DevMesh &, const DevTables &,
                                       const StatScales &, const StatBuffers &, int, cudaStream_t);
template void launch_statistic<float>(const DevParticlesT<float> &, DevCount, const DevMesh &, const DevTables &,
                                      const StatScales &, const StatBuffers &, int, cudaStream_t);

}  // namespace mcb200
