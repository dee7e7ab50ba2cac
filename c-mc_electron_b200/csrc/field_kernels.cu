// field_kernels.cu -- deposition, Poisson solve and field update on the GPU.
//
//  * deposit: MeshQuantities::compute_cell_charge (src/mcmodel.cpp:2664-2712)
//    and particle_to_density (:348-417) in one pass over the particle store,
//    summed in int64 fixed point so the result does not depend on thread
//    order.  The fixed-point unit comes from the store's charge bounds,
//    count x max |q| per carrier type (every cell or node sum is bounded by
//    it): 2^61 / bound, rounded to a power of two.
//  * Poisson: the reference factorises its FV matrix with KLU and solves it
//    every step (linear_poisson_solver, :2714-2730).  Here the Dirichlet
//    contact rows are eliminated, which leaves a symmetric positive-definite
//    system, and Jacobi-preconditioned CG iterates it in FP64 to the
//    requested relative residual.  Dot products use fixed-order two-stage
//    reductions, so a solve is bit-reproducible.
//  * pot2field (:2776-2855): cell field from the 8 corner potentials,
//    stored as felt by each carrier (ChargeSign applied).
#include <cooperative_groups.h>

#include <algorithm>

#include "device_state.cuh"
#include "field_kernels.h"
#include "poisson_common.cuh"
#include "pdl.cuh"
#include "warp_segments.cuh"

namespace mcb200 {

namespace cg = cooperative_groups;

constexpr uint32_t kDeadBit = 1u << 16;

// Per carrier type: the largest |q| (as its IEEE bit pattern, which orders
// like the value for non-negative doubles) and the particle count.  count x
// max |q| bounds every cell or node sum of that type, exactly and
// independently of thread order.  out = {max_e bits, max_h bits, n_e, n_h}.
// Warp shuffles, then one shared-memory pass per block, then one atomic
// per block and value.
__global__ void __launch_bounds__(256) charge_bounds_kernel(const double *charge, const uint32_t *meta,
                                                            DevCount count, unsigned long long *out) {
  __shared__ unsigned long long red[4][8];
  const int n = count.get();
  unsigned long long mx[2] = {0, 0}, cnt[2] = {0, 0};
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const uint32_t m = meta[p];
    if (m & kDeadBit) continue;
    const int t = ((m >> 8) & 255) == 0 ? 0 : 1;
    const unsigned long long b = (unsigned long long)__double_as_longlong(fabs(charge[p]));
    mx[t] = b > mx[t] ? b : mx[t];
    cnt[t] += 1;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int t = 0; t < 2; ++t) {
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long om = __shfl_down_sync(0xffffffffu, mx[t], o);
      mx[t] = om > mx[t] ? om : mx[t];
      cnt[t] += __shfl_down_sync(0xffffffffu, cnt[t], o);
    }
    if (lane == 0) {
      red[t][warp] = mx[t];
      red[2 + t][warp] = cnt[t];
    }
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    const int v = threadIdx.x;
    unsigned long long a = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) a = v < 2 ? (red[v][w] > a ? red[v][w] : a) : a + red[v][w];
    if (v < 2) {
      if (a) atomicMax(out + v, a);
    } else if (a) {
      atomicAdd(out + v, a);
    }
  }
}

// Fixed-point units from the bounds of charge_bounds_kernel: a sum whose
// magnitude is below 2^e gets the unit 2^(61 - e) (61 bits of range);
// empty sums get 1.  s[0]: electron cell sums, [1]: hole cell sums, [2]:
// |q| and node sums.  Every thread that needs them derives them from the
// four bound words (the store's, current before the deposition starts).
__device__ double fixed_unit(double bound) {
  if (!(bound > 0.0)) return 1.0;
  int e = 0;
  frexp(bound, &e);  // bound < 2^e
  return ldexp(1.0, 61 - e);
}
__device__ DepositScales deposit_scales(const unsigned long long *b) {
  const double qe = __longlong_as_double((long long)b[0]), qh = __longlong_as_double((long long)b[1]);
  const double be = (double)b[2] * qe, bh = (double)b[3] * qh;
  DepositScales out;
  out.s[0] = fixed_unit(be);
  out.s[1] = fixed_unit(bh);
  out.s[2] = fixed_unit(be + bh);
  return out;
}

__device__ __forceinline__ long long fx(double v, double scale) { return __double2ll_rn(v * scale); }
__device__ __forceinline__ void fx_put(long long *p, long long v) {
  atomicAdd(reinterpret_cast<unsigned long long *>(p), (unsigned long long)v);
}

// scale[0]: electron cell sums, [1]: hole cell sums, [2]: |q| and node sums.
// Lanes of a warp walk consecutive particles; runs of particles of the same
// cell and carrier type add their fixed-point terms before one atomic each.
template <typename R>
__global__ void __launch_bounds__(256) deposit_kernel(DevParticlesT<R> P, DevCount count, DevMesh M,
                                                      const unsigned long long *bounds, long long *cell_e,
                                                      long long *cell_h, long long *cell_abs, long long *node_q) {
  pdl_wait();
  const int n = count.get();
  const DepositScales S = deposit_scales(bounds);
  const int px = M.nx + 1, pz = M.nz + 1;
  const double scale = S.s[2];
  const unsigned lane = threadIdx.x & 31u;
  for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += gridDim.x * blockDim.x) {
    const int p = base + (int)lane;
    const uint32_t meta = p < n ? P.meta[p] : kDeadBit;
    const bool live = !(meta & kDeadBit);
    const uint32_t c = live ? P.cell[p] : 0u;
    const int type = ((meta >> 8) & 255) == 0 ? 0 : 1;
    const WarpRuns runs(live ? (c | ((unsigned)type << 30)) : 0xffffffffu);
    const int i = c & 1023, j = (c >> 10) & 1023, k = (c >> 20) & 1023;
    long long vc = 0, va = 0, vn[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (live) {
      const double cc = P.charge[p];
      vc = fx(cc, type == 0 ? S.s[0] : S.s[1]);
      va = fx(fabs(cc), scale);
      double rx, ry, rz;
      if constexpr (sizeof(R) == 4) {  // FP32 store: positions relative to the cell's low corner
        rx = (double)P.x[p] / M.dx[i];
        ry = (double)P.y[p] / M.dy[j];
        rz = (double)P.z[p] / M.dz[k];
      } else {
        rx = (P.x[p] - M.lx[i]) / M.dx[i];
        ry = (P.y[p] - M.ly[j]) / M.dy[j];
        rz = (P.z[p] - M.lz[k]) / M.dz[k];
      }
      vn[0] = fx(cc * (1 - ry) * (1 - rx) * (1 - rz), scale);
      vn[1] = fx(cc * (1 - ry) * rx * (1 - rz), scale);
      vn[2] = fx(cc * (1 - ry) * (1 - rx) * rz, scale);
      vn[3] = fx(cc * (1 - ry) * rx * rz, scale);
      vn[4] = fx(cc * ry * (1 - rx) * (1 - rz), scale);
      vn[5] = fx(cc * ry * rx * (1 - rz), scale);
      vn[6] = fx(cc * ry * (1 - rx) * rz, scale);
      vn[7] = fx(cc * ry * rx * rz, scale);
    }
    const long long sc = runs.sum(vc), sa = runs.sum(va);
    long long sn[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) sn[q] = runs.sum(vn[q]);
    if (live && runs.tail) {
      const int cell = (j * M.nx + i) * M.nz + k;
      fx_put((type == 0 ? cell_e : cell_h) + cell, sc);
      fx_put(cell_abs + cell, sa);
      auto node = [&](int a, int b, int d) { return node_q + ((size_t)b * px + a) * pz + d; };
      fx_put(node(i, j, k), sn[0]);
      fx_put(node(i + 1, j, k), sn[1]);
      fx_put(node(i, j, k + 1), sn[2]);
      fx_put(node(i + 1, j, k + 1), sn[3]);
      fx_put(node(i, j + 1, k), sn[4]);
      fx_put(node(i + 1, j + 1, k), sn[5]);
      fx_put(node(i, j + 1, k + 1), sn[6]);
      fx_put(node(i + 1, j + 1, k + 1), sn[7]);
    }
  }
}

// compute_cell_charge's final loop (:2705-2710) with the per-cell sums, and
// particle_to_density's volume division (:408-416), in one pass: thread t
// takes cell t and node t.  It clears the fixed-point sums it reads, so the
// next deposition starts from zero without a memset.
__global__ void deposit_sums_kernel(int cells, int nodes, const unsigned long long *bounds, long long *cell_e,
                                    long long *cell_h, long long *cell_abs, const double *cvol, const double *da,
                                    double *e_out, double *h_out, double *rho_out, long long *node_q,
                                    const double *pvol, double *density) {
  pdl_wait();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= cells && t >= nodes) return;
  const DepositScales S = deposit_scales(bounds);
  if (t < cells) {
    e_out[t] = (double)cell_e[t] / S.s[0];
    h_out[t] = (double)cell_h[t] / S.s[1];
    const double r = (double)cell_abs[t] / S.s[2] / cvol[t];
    const double half = 0.5 * da[t];
    rho_out[t] = r > half ? r : half;
    cell_e[t] = 0;
    cell_h[t] = 0;
    cell_abs[t] = 0;
  }
  if (t < nodes) {
    const double q = (double)node_q[t] / S.s[2];
    density[t] = fabs(pvol[t]) > 0 ? q / pvol[t] : q;
    node_q[t] = 0;
  }
}

// compute_rhs, src/mcmodel.cpp:2858-2893.
__global__ void rhs_kernel(int nodes, const double *density, const double *pvol, const double *pdop,
                           const uint8_t *dirichlet, const double *vapp, const double *vadd, const double *phims,
                           double *rhs) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nodes) return;
  if (dirichlet[p]) rhs[p] = vapp[p] + vadd[p] + phims[p];
  else rhs[p] = fabs(density[p]) > 0 ? density[p] * pvol[p] + pdop[p] : 0.0;
}


// y = A_ff x on free nodes (Dirichlet neighbours excluded); Dirichlet rows: y = 0.
// With `rhs`, writes b_ff - A x instead, where b_ff folds the Dirichlet values
// into the free rows (elimination of the contact rows).
__global__ void stencil_apply(int nodes, Grid3 g, const double *st, const uint8_t *dir, const double *x,
                              const double *rhs, double *y) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nodes) return;
  if (dir[p]) {
    y[p] = 0.0;
    return;
  }
  int i, j, k;
  node_ijk(p, g, i, j, k);
  const double *a = st + (size_t)p * 7;
  double acc = a[6] * x[p];
  double fold = 0.0;  // contributions of Dirichlet neighbours (known values)
  const int nb[6] = {i > 0 ? p - g.pz : -1, i + 1 < g.px ? p + g.pz : -1, j > 0 ? p - g.px * g.pz : -1,
                     j + 1 < g.py ? p + g.px * g.pz : -1, k > 0 ? p - 1 : -1, k + 1 < g.pz ? p + 1 : -1};
#pragma unroll
  for (int s = 0; s < 6; ++s) {
    const int q = nb[s];
    if (q < 0 || a[s] == 0.0) continue;
    if (dir[q]) fold += a[s] * x[q];
    else acc += a[s] * x[q];
  }
  y[p] = rhs ? (rhs[p] - fold) - acc : acc;
}


constexpr int kRedGrid = 296;  // 2 x 148 SMs; fixed so the reduction order is fixed

__global__ void __launch_bounds__(kRedBlock) dot_partial(int n, const double *a, const double *b, double *part) {
  double v = 0.0;
  for (int i = blockIdx.x * kRedBlock + threadIdx.x; i < n; i += kRedGrid * kRedBlock) v += a[i] * b[i];
  const double s = block_sum<kRedBlock>(v);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}
__global__ void __launch_bounds__(kRedBlock) dot_final(const double *part, double *out) {
  double v = 0.0;
  for (int i = threadIdx.x; i < kRedGrid; i += kRedBlock) v += part[i];
  const double s = block_sum<kRedBlock>(v);
  if (threadIdx.x == 0) *out = s;
}

// CG scalars in device memory: [0] rz, [3] rr, [6] ||b||^2, [7] converged,
// [8] iterations, [9] (rel_tol ||b||)^2
__global__ void cg_init(int n, const double *r, const double *diag_inv, double *z, double *p, const uint8_t *dir,
                        const double *rhs, double *x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (dir[i]) {
    x[i] = rhs[i];
    z[i] = 0.0;
    p[i] = 0.0;
    return;
  }
  z[i] = r[i] * diag_inv[i];
  p[i] = z[i];
}
// Free-row right-hand side with the Dirichlet values folded in (for ||b||).
__global__ void folded_rhs(int nodes, Grid3 g, const double *st, const uint8_t *dir, const double *rhs, double *b) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nodes) return;
  if (dir[p]) {
    b[p] = 0.0;
    return;
  }
  int i, j, k;
  node_ijk(p, g, i, j, k);
  const double *a = st + (size_t)p * 7;
  double fold = 0.0;
  const int nb[6] = {i > 0 ? p - g.pz : -1, i + 1 < g.px ? p + g.pz : -1, j > 0 ? p - g.px * g.pz : -1,
                     j + 1 < g.py ? p + g.px * g.pz : -1, k > 0 ? p - 1 : -1, k + 1 < g.pz ? p + 1 : -1};
  for (int s = 0; s < 6; ++s)
    if (nb[s] >= 0 && a[s] != 0.0 && dir[nb[s]]) fold += a[s] * rhs[nb[s]];
  b[p] = rhs[p] - fold;
}
__global__ void set_dirichlet(int nodes, const uint8_t *dir, const double *rhs, double *x) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < nodes && dir[p]) x[p] = rhs[p];
}

// ---- persistent CG -----------------------------------------------------------
// One cooperative launch runs every iteration of a solve.  Per iteration two
// grid-wide barriers: (A) p_new = z + beta p_old, computed on the fly for the
// node and its neighbours (p ping-pongs between two buffers), q = A p_new and
// the block partials of p.q; (B) alpha, the x / r / z update and the
// partials of r.z and r.r.  After each barrier every block sums all partials
// itself, in the same fixed order, so every block takes the same scalars and
// the same convergence decision, and a solve is bit-reproducible for a given
// grid.

__global__ void __launch_bounds__(kRedBlock) cg_persistent(int nodes, Grid3 g, const double *st, const uint8_t *dir,
                                                           const double *diag_inv, double *x, double *r, double *z,
                                                           double *p0, double *p1, double *q, double *part,
                                                           double *sc, int max_iter) {
  cg::grid_group grid = cg::this_grid();
  const int nblk = gridDim.x;
  double *part_pq = part, *part_rz = part + nblk, *part_rr = part + 2 * nblk;
  double rz = sc[0], rr = sc[3], beta = 0.0;  // p0 holds z: the first p is z
  const double tol2 = sc[9];
  bool done = sc[7] != 0.0;
  int it = 0;
  const double *pin = p0;
  double *pout = p1;
  const int stride = nblk * kRedBlock;
  while (!done && it < max_iter) {
    double v = 0.0;
    for (int n = blockIdx.x * kRedBlock + threadIdx.x; n < nodes; n += stride) {
      if (dir[n]) {
        q[n] = 0.0;
        pout[n] = 0.0;
        continue;
      }
      int i, j, k;
      node_ijk(n, g, i, j, k);
      const double *a = st + (size_t)n * 7;
      const double pn = z[n] + beta * pin[n];
      pout[n] = pn;
      double acc = a[6] * pn;
      const int nb[6] = {i > 0 ? n - g.pz : -1, i + 1 < g.px ? n + g.pz : -1, j > 0 ? n - g.px * g.pz : -1,
                         j + 1 < g.py ? n + g.px * g.pz : -1, k > 0 ? n - 1 : -1, k + 1 < g.pz ? n + 1 : -1};
#pragma unroll
      for (int s = 0; s < 6; ++s) {
        const int m = nb[s];
        if (m < 0 || a[s] == 0.0 || dir[m]) continue;
        acc += a[s] * (z[m] + beta * pin[m]);
      }
      q[n] = acc;
      v += pn * acc;
    }
    const double bs = block_sum<kRedBlock>(v);
    if (threadIdx.x == 0) part_pq[blockIdx.x] = bs;
    grid.sync();
    const double alpha = rz / sum_partials(part_pq, nblk);
    double a1 = 0.0, a2 = 0.0;
    for (int n = blockIdx.x * kRedBlock + threadIdx.x; n < nodes; n += stride) {
      if (dir[n]) continue;
      x[n] += alpha * pout[n];
      const double rn = r[n] - alpha * q[n];
      r[n] = rn;
      const double zn = rn * diag_inv[n];
      z[n] = zn;
      a1 += rn * zn;
      a2 += rn * rn;
    }
    const double b1 = block_sum<kRedBlock>(a1);
    const double b2 = block_sum<kRedBlock>(a2);
    if (threadIdx.x == 0) {
      part_rz[blockIdx.x] = b1;
      part_rr[blockIdx.x] = b2;
    }
    grid.sync();
    const double rz_new = sum_partials(part_rz, nblk);
    rr = sum_partials(part_rr, nblk);
    beta = rz_new / rz;
    rz = rz_new;
    ++it;
    done = rr <= tol2;
    const double *t = pout;
    pout = const_cast<double *>(pin);
    pin = t;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sc[0] = rz;
    sc[3] = rr;
    sc[8] = it;
  }
}

// Running solve statistics: st[0] solves, st[1] iterations, st[2] the
// largest relative true residual.  sc[3] holds the final ||b - Ax||^2 and
// sc[6] ||b||^2.
__global__ void poisson_stats_kernel(const double *sc, double *st) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double bnorm = sqrt(sc[6]) > 0 ? sqrt(sc[6]) : 1.0;
  st[0] += 1.0;
  st[1] += sc[8];
  st[2] = fmax(st[2], sqrt(sc[3]) / bnorm);
}

// sc[9] = (rel_tol * ||b||)^2; converged already when the warm start meets it
__global__ void cg_setup(double *sc, double rel_tol2) {
  sc[9] = rel_tol2 * sc[6];
  sc[7] = sc[3] <= sc[9] ? 1.0 : 0.0;
  sc[8] = 0.0;
}

// pot2field / pot2field_for_hole, src/mcmodel.cpp:2732-2855: the field of
// each cell from the averaged edge differences of its corner potentials,
// stored as felt.  Holes take it from the Poisson potential, electrons from
// pot_e: the same potential, or the quantum-corrected one (compute_field,
// :2240-2262).
__global__ void pot2field_kernel(DevMesh M, const double *pot, const double *pot_e, double *efield, double *hfield) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int cells = M.nx * M.ny * M.nz;
  if (c >= cells) return;
  const int k = c % M.nz, t = c / M.nz, i = t % M.nx, j = t / M.nx;
  const int px = M.nx + 1, pz = M.nz + 1;
  auto field = [&](const double *v, double &fx, double &fy, double &fz) {
    auto P = [&](int a, int b, int d) { return v[((size_t)b * px + a) * pz + d]; };
    fx = -(P(i + 1, j, k) - P(i, j, k) + P(i + 1, j + 1, k) - P(i, j + 1, k) + P(i + 1, j, k + 1) - P(i, j, k + 1) +
           P(i + 1, j + 1, k + 1) - P(i, j + 1, k + 1)) / (4.0 * M.dx[i]);
    fy = -(P(i, j + 1, k) + P(i + 1, j + 1, k) + P(i, j + 1, k + 1) + P(i + 1, j + 1, k + 1) - P(i, j, k) -
           P(i + 1, j, k) - P(i, j, k + 1) - P(i + 1, j, k + 1)) / (4.0 * M.dy[j]);
    fz = -(P(i, j, k + 1) + P(i + 1, j, k + 1) + P(i, j + 1, k + 1) + P(i + 1, j + 1, k + 1) - P(i, j, k) -
           P(i + 1, j, k) - P(i, j + 1, k) - P(i + 1, j + 1, k)) / (4.0 * M.dz[k]);
  };
  double fx, fy, fz;
  field(pot, fx, fy, fz);
  // ChargeSign = {-1, +1} (src/Constant_GlobalVariable_MathFunction.cpp:18)
  hfield[3 * (size_t)c + 0] = fx;
  hfield[3 * (size_t)c + 1] = fy;
  hfield[3 * (size_t)c + 2] = fz;
  if (pot_e != pot) field(pot_e, fx, fy, fz);
  efield[3 * (size_t)c + 0] = -1.0 * fx;
  efield[3 * (size_t)c + 1] = -1.0 * fy;
  efield[3 * (size_t)c + 2] = -1.0 * fz;
}

// ---------------------------------------------------------------------------
static inline int blocks(long long n, int b) { return (int)((n + b - 1) / b); }

template <typename R>
void launch_charge_bounds(const DevParticlesT<R> &P, DevCount n, unsigned long long *out, int grid, cudaStream_t s) {
  cudaMemsetAsync(out, 0, 4 * sizeof(unsigned long long), s);
  charge_bounds_kernel<<<grid, 256, 0, s>>>(P.charge, P.meta, n, out);
}

template <typename R>
void launch_deposit(const DevParticlesT<R> &P, DevCount n, const DevMesh &M, const FieldBuffers &f, int grid,
                    cudaStream_t s) {
  const int cells = M.nx * M.ny * M.nz, nodes = (M.nx + 1) * (M.ny + 1) * (M.nz + 1);
  launch_pdl(deposit_kernel<R>, grid, 256, 0, s, P, n, M, (const unsigned long long *)f.abs_sum, f.acc_cell,
             f.acc_cell + cells, f.acc_cell + 2 * (size_t)cells, f.acc_node);
  launch_pdl(deposit_sums_kernel, blocks(std::max(cells, nodes), 256), 256, 0, s, cells, nodes,
             (const unsigned long long *)f.abs_sum, f.acc_cell, f.acc_cell + cells, f.acc_cell + 2 * (size_t)cells,
             (const double *)f.cvol, M.da, f.cell_e, f.cell_h, const_cast<double *>(M.rho), f.acc_node,
             (const double *)f.pvol, f.density);
}

template void launch_charge_bounds<double>(const DevParticlesT<double> &, DevCount, unsigned long long *, int,
                                           cudaStream_t);
template void launch_charge_bounds<float>(const DevParticlesT<float> &, DevCount, unsigned long long *, int,
                                          cudaStream_t);
template void launch_deposit<double>(const DevParticlesT<double> &, DevCount, const DevMesh &, const FieldBuffers &,
                                     int, cudaStream_t);
template void launch_deposit<float>(const DevParticlesT<float> &, DevCount, const DevMesh &, const FieldBuffers &,
                                    int, cudaStream_t);

void launch_rhs(int nodes, const FieldBuffers &f, cudaStream_t s) {
  rhs_kernel<<<blocks(nodes, 256), 256, 0, s>>>(nodes, f.density, f.pvol, f.pdop, f.dirichlet, f.bc_vapp, f.vadd,
                                                 f.bc_phims, f.rhs);
}

static void dot(int n, const double *a, const double *b, double *part, double *out, cudaStream_t s) {
  dot_partial<<<kRedGrid, kRedBlock, 0, s>>>(n, a, b, part);
  dot_final<<<1, kRedBlock, 0, s>>>(part, out);
}

int cg_prepare(const DevMesh &M, const FieldBuffers &f, double rel_tol, cudaStream_t s, CgPlan &plan) {
  const int nodes = (M.nx + 1) * (M.ny + 1) * (M.nz + 1);
  const Grid3 g{M.nx + 1, M.ny + 1, M.nz + 1};
  const int nb = blocks(nodes, 256);
  const bool use_mg = f.mg && plan.method != kCgJacobi;
  if (plan.method == kCgMultigrid && !f.mg) return 1;
  double *sc = f.cg_scalars;
  plan.rel_tol2 = rel_tol * rel_tol;
  if (!use_mg) {  // the multigrid launch does its own set-up
    // ||b_free|| with the Dirichlet values folded in
    set_dirichlet<<<nb, 256, 0, s>>>(nodes, f.dirichlet, f.rhs, f.potential);
    folded_rhs<<<nb, 256, 0, s>>>(nodes, g, f.stencil, f.dirichlet, f.rhs, f.cg_q);
    dot(nodes, f.cg_q, f.cg_q, f.cg_part, sc + 6, s);
    // r = b - A x (x: the previous potential, a warm start)
    stencil_apply<<<nb, 256, 0, s>>>(nodes, g, f.stencil, f.dirichlet, f.potential, f.rhs, f.cg_r);
    cg_init<<<nb, 256, 0, s>>>(nodes, f.cg_r, f.diag_inv, f.cg_z, f.cg_p, f.dirichlet, f.rhs, f.potential);
    dot(nodes, f.cg_r, f.cg_z, f.cg_part, sc + 0, s);
    dot(nodes, f.cg_r, f.cg_r, f.cg_part, sc + 3, s);
    cg_setup<<<1, 1, 0, s>>>(sc, plan.rel_tol2);
  }
  // the persistent launch's grid, fixed per context (so is the reduction order)
  if (plan.grid == 0 || plan.used != (use_mg ? kCgMultigrid : kCgJacobi)) {
    int dev = 0, sms = 0, per_sm = 0, coop = 0, most = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    if (use_mg) {
      most = cg_mg_max_grid();
    } else if (coop &&
               cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cg_persistent, kRedBlock, 0) == cudaSuccess) {
      most = per_sm * sms;
    }
    if (most < 1) return 1;
    most = std::min(most, kCgMaxGrid);
    // the V-cycle's short phases are barrier-bound: one 512-thread block
    // per SM measured fastest on the FinFET mesh (fewer blocks arrive at
    // each barrier; more would idle on its coarse levels)
    const int fallback = use_mg ? std::min(most, cg_mg_blocks_per_sm() * sms) : most;
    plan.grid = plan.blocks > 0 ? std::min(plan.blocks, most) : fallback;
    plan.used = use_mg ? kCgMultigrid : kCgJacobi;
  }
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

MgSystem cg_mg_system(const DevMesh &M, const FieldBuffers &f, int max_iter, double rel_tol2) {
  MgSystem y;
  y.mg = *f.mg;
  y.mg.L[0].b = f.cg_r;
  y.mg.L[0].xa = f.cg_z;
  y.st7 = f.stencil;
  y.dirichlet = f.dirichlet;
  y.x = f.potential; y.r = f.cg_r; y.r1 = f.cg_r1; y.p0 = f.cg_p; y.p1 = f.cg_p1; y.q = f.cg_q; y.part = f.cg_part;
  y.sc = f.cg_scalars;
  y.rhs = f.rhs;
  y.stats = f.poisson_stats;
  y.rel_tol2 = rel_tol2;
  y.px = M.nx + 1; y.py = M.ny + 1; y.pz = M.nz + 1;
  y.max_iter = max_iter;
  return y;
}

int cg_launch(const DevMesh &M, const FieldBuffers &f, int max_iter, cudaStream_t s, CgPlan &plan) {
  const int nodes = (M.nx + 1) * (M.ny + 1) * (M.nz + 1);
  const Grid3 g{M.nx + 1, M.ny + 1, M.nz + 1};
  double *x = f.potential, *r = f.cg_r, *z = f.cg_z, *p0 = f.cg_p, *p1 = f.cg_p1, *q = f.cg_q, *part = f.cg_part;
  double *sc = f.cg_scalars;
  if (plan.used == kCgMultigrid) {
    if (launch_cg_mg(cg_mg_system(M, f, max_iter, plan.rel_tol2), plan.grid, s) != cudaSuccess) return 1;
  } else {
    int nodes_arg = nodes, max_arg = max_iter;
    Grid3 g_arg = g;
    const double *st = f.stencil, *dinv = f.diag_inv;
    const uint8_t *dirp = f.dirichlet;
    void *args[] = {&nodes_arg, &g_arg, &st, &dirp, &dinv, &x, &r, &z, &p0, &p1, &q, &part, &sc, &max_arg};
    if (cudaLaunchCooperativeKernel((const void *)cg_persistent, plan.grid, kRedBlock, args, 0, s) != cudaSuccess)
      return 1;
  }
  plan.launches += 1;
  return 0;
}

int cg_finish(const DevMesh &M, const FieldBuffers &f, const CgPlan &plan, cudaStream_t s, double *host_scratch,
              int *iterations, double *rel_residual) {
  const int nodes = (M.nx + 1) * (M.ny + 1) * (M.nz + 1);
  const int nb = blocks(nodes, 256);
  double *sc = f.cg_scalars;
  if (plan.used != kCgMultigrid) {  // (the multigrid launch ends with both)
    // true residual of the final iterate, and the running statistics
    stencil_apply<<<nb, 256, 0, s>>>(nodes, Grid3{M.nx + 1, M.ny + 1, M.nz + 1}, f.stencil, f.dirichlet,
                                     f.potential, f.rhs, f.cg_r);
    dot(nodes, f.cg_r, f.cg_r, f.cg_part, sc + 3, s);
    poisson_stats_kernel<<<1, 32, 0, s>>>(sc, f.poisson_stats);
  }
  if (!iterations && !rel_residual) return cudaGetLastError() == cudaSuccess ? 0 : 1;  // nothing waits
  cudaMemcpyAsync(host_scratch, sc, 10 * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return 1;
  const double bnorm = sqrt(host_scratch[6]) > 0 ? sqrt(host_scratch[6]) : 1.0;
  if (iterations) *iterations = (int)host_scratch[8];
  if (rel_residual) *rel_residual = sqrt(host_scratch[3]) / bnorm;
  return 0;
}

int cg_solve(const DevMesh &M, const FieldBuffers &f, double rel_tol, int max_iter, cudaStream_t s,
             double *host_scratch, int *iterations, double *rel_residual, CgPlan &plan) {
  if (cg_prepare(M, f, rel_tol, s, plan) || cg_launch(M, f, max_iter, s, plan)) return 1;
  return cg_finish(M, f, plan, s, host_scratch, iterations, rel_residual);
}

void launch_pot2field(const DevMesh &M, const double *pot, cudaStream_t s, const double *pot_e) {
  const int cells = M.nx * M.ny * M.nz;
  pot2field_kernel<<<blocks(cells, 256), 256, 0, s>>>(M, pot, pot_e ? pot_e : pot, const_cast<double *>(M.efield),
                                                        const_cast<double *>(M.hfield));
}

}  // namespace mcb200
