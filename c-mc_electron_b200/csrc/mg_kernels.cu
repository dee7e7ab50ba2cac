// mg_kernels.cu -- conjugate gradients preconditioned by one geometric
// multigrid V-cycle, every iteration of a solve in one cooperative launch.
//
// The reference factorises its finite-volume Poisson matrix with KLU and
// solves it every step (MeshQuantities::linear_poisson_solver,
// src/mcmodel.cpp:2714-2730).  Here the Dirichlet contact rows are
// eliminated and the remaining SPD system is solved by CG in FP64 to a
// relative residual; the preconditioner is a symmetric V-cycle over the
// hierarchy of mg_setup.h: damped Jacobi (nu sweeps before and after the
// coarse correction, weight 1.6 / rho(D^-1 A) per level), residual
// restriction by P^T (gather over the 3 x 3 x 3 fine neighbourhood of each
// coarse node), the exact dense inverse on the coarsest level, trilinear
// prolongation.  Every phase is a grid-stride pass over one level's nodes
// separated by grid-wide barriers; nothing is accumulated with atomics and
// the dot products use fixed-order reductions, so a solve is
// bit-reproducible for a given grid.
#include <cooperative_groups.h>

#include <algorithm>
#include <stdexcept>

#include "mg_kernels.h"
#include "poisson_common.cuh"

namespace mcb200 {

namespace cg = cooperative_groups;

namespace {

// Threads per block of the solve kernels and blocks per SM of the default
// grid (tuning defines).  With at most 64 registers a thread (1024 threads
// of registers per SM), kMgBlock x 1024 / kMgBlock blocks fill the SM.
// Measured on the FinFET solve (same 75,776 threads): one 512-thread block
// per SM 3 % faster than two of 256 (half the blocks arrive at each grid
// barrier); 1024 threads on one block per SM, or 512 x 2, slower.
#ifndef MCB200_MG_BLOCK
#define MCB200_MG_BLOCK 512
#endif
#ifndef MCB200_MG_BLOCKS_PER_SM
#define MCB200_MG_BLOCKS_PER_SM 1
#endif
constexpr int kMgBlock = MCB200_MG_BLOCK;
static_assert(kMgBlock % 32 == 0 && 1024 % kMgBlock == 0, "MCB200_MG_BLOCK: 32-1024, dividing 1024");

#ifdef MCB200_MG_TRACE
// Opt-in phase trace (build with -DMCB200_MG_TRACE): block 0 records
// (phase id, %globaltimer) after every barrier of the first solve.
constexpr int kTraceMax = 8192;
__device__ unsigned long long g_trace[2 * kTraceMax];
__device__ int g_trace_n;
__device__ __forceinline__ void trace(int id) {
  if (blockIdx.x == 0 && threadIdx.x == 0 && g_trace_n < kTraceMax) {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    g_trace[2 * g_trace_n] = id;
    g_trace[2 * g_trace_n + 1] = t;
    ++g_trace_n;
  }
}
#else
__device__ __forceinline__ void trace(int) {}
#endif

// The coefficients of node n in a level's stencil, stored coefficient-major
// ([coefficient][node], `stride` nodes): the lanes of a warp, on consecutive
// nodes, read consecutive doubles for each coefficient.
struct CoefRow {
  const double *st;
  int stride;
  __device__ __forceinline__ double operator[](int t) const { return st[(size_t)t * stride]; }
};

// (A x)[n] with the 7-point stencil of the CG (-x, +x, -y, +y, -z, +z,
// diagonal).  x is zero on Dirichlet nodes and isolated nodes have no
// couplings, so no neighbour needs masking.  A coefficient towards a
// neighbour off the grid is zero (the finite-volume assembly adds only
// in-grid couplings), so an off-grid neighbour's index is clamped to the
// node itself: every load is unconditional and independent, and the exact
// zero products leave the sum as the branchy form would make it.
__device__ __forceinline__ double apply7(const double *st7, const Grid3 &g, const double *x, int n) {
  int i, j, k;
  node_ijk(n, g, i, j, k);
  const CoefRow a{st7 + n, g.px * g.py * g.pz};
  const int sx = g.pz, sy = g.px * g.pz;
  double acc = a[6] * x[n];
  acc += a[0] * x[i > 0 ? n - sx : n];
  acc += a[1] * x[i + 1 < g.px ? n + sx : n];
  acc += a[2] * x[j > 0 ? n - sy : n];
  acc += a[3] * x[j + 1 < g.py ? n + sy : n];
  acc += a[4] * x[k > 0 ? n - 1 : n];
  acc += a[5] * x[k + 1 < g.pz ? n + 1 : n];
  return acc;
}

// Lanes that share one node of a level of n nodes, with `stride` threads on
// the level: 8, 4 or 2 where every group still gets a node, else 1.  The
// coarse levels have far fewer nodes than the grid has threads; splitting
// a node's 27 couplings over a group puts more independent loads in flight
// per node and shortens the pass, which is latency-bound.
__device__ __forceinline__ int lanes_per_node(int n, int stride) {
  return n * 8 <= stride ? 8 : n * 4 <= stride ? 4 : n * 2 <= stride ? 2 : 1;
}

// Sum over an aligned group of G lanes of a warp; every lane of the group
// gets the same bits (a butterfly adds the same two operands on both sides).
template <int G>
__device__ __forceinline__ double group_sum(double v) {
  if constexpr (G > 1) {
    const unsigned lane = threadIdx.x & 31u;
    const unsigned mask = ((1u << G) - 1u) << (lane & ~(unsigned)(G - 1));
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o);
  }
  return v;
}

// Lane g's share of (A x)[n] with a level's 27-point Galerkin stencil,
// entry ((di+1)*3 + (dj+1))*3 + (dk+1): the (di, dj) rows g, g + G, ...
// (all nine, in order, for G = 1).  Off-grid couplings are zero (the
// Galerkin product couples existing coarse nodes only), so off-grid
// indices are clamped as in apply7.
template <int G>
__device__ __forceinline__ double apply27_part(const MgDevLevel &L, const double *x, int n, int g) {
  int i, j, k;
  node_ijk(n, Grid3{L.px, L.py, L.pz}, i, j, k);
  const CoefRow a{L.st + n, L.n};
  const int km = k > 0 ? -1 : 0, kp = k + 1 < L.pz ? 1 : 0;
  double acc = 0.0;
#pragma unroll
  for (int t = 0; t < (9 + G - 1) / G; ++t) {
    const int row = g + t * G;
    if (row < 9) {
      const int i2 = min(max(i + row / 3 - 1, 0), L.px - 1), j2 = min(max(j + row % 3 - 1, 0), L.py - 1);
      const int base = (j2 * L.px + i2) * L.pz + k;
      acc += a[row * 3] * x[base + km];
      acc += a[row * 3 + 1] * x[base];
      acc += a[row * 3 + 2] * x[base + kp];
    }
  }
  return acc;
}

struct Solve {
  const MgDevice &mg;
  const double *st7;
  Grid3 g0;
  int tid, stride;
  unsigned cur;      // bit l: level l's iterate is in xb (else xa)
  const double *b0;  // level 0's right side: the CG residual buffer of this iteration

  __device__ double *X(int l) const { return (cur >> l) & 1u ? mg.L[l].xb : mg.L[l].xa; }
  __device__ double *Xo(int l) const { return (cur >> l) & 1u ? mg.L[l].xa : mg.L[l].xb; }
  // First sweep from a zero iterate: x = omega D^-1 b (level 0's isolated
  // rows: D^-1 b), for node n.
  __device__ void first(int l, int n, double b) const {
    const MgDevLevel &L = mg.L[l];
    X(l)[n] = L.dir[n] ? (l == 0 ? L.dinv[n] * b : 0.0) : L.omega * L.dinv[n] * b;
  }
  // One damped-Jacobi sweep into the other buffer; returns sum b.x_new of
  // this thread's nodes when `dot`.  Level 0 one node a thread (7-point);
  // a coarser level G lanes a node (lanes_per_node), lane 0 writing.
  template <int G>
  __device__ double sweep_level(int l, bool dot) const {
    const MgDevLevel &L = mg.L[l];
    const double *xc = X(l), *b = l == 0 ? b0 : L.b;
    double *xn = Xo(l);
    const int g = tid % G;
    double acc = 0.0;
    for (int n = tid / G; n < L.n; n += stride / G) {
      const double ax = l == 0 ? apply7(st7, g0, xc, n) : group_sum<G>(apply27_part<G>(L, xc, n, g));
      if (g != 0) continue;
      const double bn = b[n], dn = L.dinv[n], xn0 = xc[n];
      double v = xn0 + L.omega * dn * (bn - ax);
      if (L.dir[n]) v = l == 0 ? dn * bn : 0.0;
      xn[n] = v;
      if (dot) acc += bn * v;
    }
    return acc;
  }
  __device__ double sweep(int l, bool dot) {
    const int G = l == 0 ? 1 : lanes_per_node(mg.L[l].n, stride);
    const double acc = G == 8   ? sweep_level<8>(l, dot)
                       : G == 4 ? sweep_level<4>(l, dot)
                       : G == 2 ? sweep_level<2>(l, dot)
                                : sweep_level<1>(l, dot);
    cur ^= 1u << l;
    return acc;
  }
  template <int G>
  __device__ void residual_level(int l) const {
    const MgDevLevel &L = mg.L[l];
    const double *x = X(l);
    const int g = tid % G;
    for (int n = tid / G; n < L.n; n += stride / G) {
      const double ax = l == 0 ? apply7(st7, g0, x, n) : group_sum<G>(apply27_part<G>(L, x, n, g));
      if (g != 0) continue;
      const double v = (l == 0 ? b0 : L.b)[n] - ax;
      L.r[n] = L.dir[n] ? 0.0 : v;
    }
  }
  __device__ void residual(int l) const {
    const int G = l == 0 ? 1 : lanes_per_node(mg.L[l].n, stride);
    if (G == 8) residual_level<8>(l);
    else if (G == 4) residual_level<4>(l);
    else if (G == 2) residual_level<2>(l);
    else residual_level<1>(l);
  }
  // b_{l+1} = P^T r_l, and the first sweep of level l+1 unless it is the
  // coarsest.  The 27 taps of a coarse node are the products of its three
  // per-axis tap triples; off-grid taps have weight 0 and a clamped index,
  // so every load is independent of the others.  G lanes a coarse node
  // (lanes_per_node), each the (x, y) tap rows g, g + G, ... of the nine.
  template <int G>
  __device__ void restrict_level(int l) const {
    const MgDevLevel &F = mg.L[l], &C = mg.L[l + 1];
    const bool smooth = l + 2 < mg.levels;
    const Grid3 gc{C.px, C.py, C.pz};
    const int g = tid % G;
    for (int c = tid / G; c < C.n; c += stride / G) {
      int ci, cj, ck;
      node_ijk(c, gc, ci, cj, ck);
      const int fi = F.keep[0][ci], fj = F.keep[1][cj], fk = F.keep[2][ck];
      double wz[3];
      int kz[3];
#pragma unroll
      for (int t = 0; t < 3; ++t) {
        wz[t] = F.rtap[2][3 * ck + t];
        kz[t] = min(max(fk - 1 + t, 0), F.pz - 1);
      }
      double acc = 0.0;
#pragma unroll
      for (int t = 0; t < (9 + G - 1) / G; ++t) {
        const int row = g + t * G;
        if (row < 9) {
          const int b = row / 3, a = row % 3;
          const double wab = F.rtap[0][3 * ci + a] * F.rtap[1][3 * cj + b];
          const int ix = min(max(fi - 1 + a, 0), F.px - 1), jy = min(max(fj - 1 + b, 0), F.py - 1);
          const double *frow = F.r + (jy * F.px + ix) * F.pz;
#pragma unroll
          for (int d = 0; d < 3; ++d) acc += wab * wz[d] * frow[kz[d]];
        }
      }
      acc = group_sum<G>(acc);
      if (g != 0) continue;
      if (C.dir[c]) acc = 0.0;
      C.b[c] = acc;
      if (smooth) first(l + 1, c, acc);
    }
  }
  __device__ void restrict_to(int l) const {
    const int G = lanes_per_node(mg.L[l + 1].n, stride);
    if (G == 8) restrict_level<8>(l);
    else if (G == 4) restrict_level<4>(l);
    else if (G == 2) restrict_level<2>(l);
    else restrict_level<1>(l);
  }
  // x_l += P x_{l+1} on the free rows.
  __device__ void prolong(int l) const {
    const MgDevLevel &F = mg.L[l], &C = mg.L[l + 1];
    const double *xc = X(l + 1);
    double *x = X(l);
    const Grid3 gf{F.px, F.py, F.pz};
    for (int n = tid; n < F.n; n += stride) {
      if (F.dir[n]) continue;
      int i, j, k;
      node_ijk(n, gf, i, j, k);
      const int2 cx = F.cmap[0][i], cy = F.cmap[1][j], cz = F.cmap[2][k];
      const double2 wx = F.wmap[0][i], wy = F.wmap[1][j], wz = F.wmap[2][k];
      double acc = 0.0;
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        const double wb = b ? wy.y : wy.x;
        if (wb == 0.0) continue;
        const int cj = b ? cy.y : cy.x;
#pragma unroll
        for (int a = 0; a < 2; ++a) {
          const double wa = a ? wx.y : wx.x;
          if (wa == 0.0) continue;
          const int ci = a ? cx.y : cx.x;
#pragma unroll
          for (int d = 0; d < 2; ++d) {
            const double wd = d ? wz.y : wz.x;
            if (wd == 0.0) continue;
            const int ck = d ? cz.y : cz.x;
            acc += wa * wb * wd * xc[(cj * C.px + ci) * C.pz + ck];
          }
        }
      }
      x[n] += acc;
    }
  }
  // x = C^-1 b on the coarsest level, one warp per row; returns sum b.x of
  // the rows this thread's warp finished (lane 0 only).
  __device__ double dense(int l) const {
    const MgDevLevel &L = mg.L[l];
    const int lane = threadIdx.x & 31, warp = tid >> 5, warps = stride >> 5;
    double *x = X(l);
    double acc = 0.0;
    for (int row = warp; row < L.n; row += warps) {
      const double *m = mg.coarse_inv + (size_t)row * L.n;
      double s = 0.0;
      for (int c = lane; c < L.n; c += 32) s += m[c] * L.b[c];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (lane == 0) {
        x[row] = s;
        acc += L.b[row] * s;
      }
    }
    return acc;
  }

  // z = M r.  On entry level 0's first sweep is in X(0) (levels > 1), and
  // with `have_r0` level 0's residual of it too (the CG update computes it,
  // one grid barrier fewer); on exit X(0) holds z, part_rz the block
  // partials of r.z (block vb of the solve), and the grid has synchronised.
  // Without `work` only the grid barriers are taken (a block of a finished
  // solve sharing the launch).
  __device__ void vcycle(cg::grid_group &grid, double *part_rz, int vb, bool work, bool have_r0) {
    const int L = mg.levels;
    double rz = 0.0;
    if (L == 1) {
      if (work) rz = dense(0);
    } else {
      for (int l = 0; l + 1 < L; ++l) {
        for (int s = 1; s < mg.nu; ++s) {
          if (work) sweep(l, false);
          grid.sync();
          trace(10 * l + 1);
        }
        if (l > 0 || !have_r0) {
          if (work) residual(l);
          grid.sync();
          trace(10 * l + 2);
        }
        if (work) restrict_to(l);
        grid.sync();
        trace(10 * l + 3);
      }
      if (work) dense(L - 1);
      grid.sync();
      trace(10 * (L - 1) + 4);
      for (int l = L - 2; l >= 0; --l) {
        if (work) prolong(l);
        grid.sync();
        trace(10 * l + 5);
        for (int s = 0; s < mg.nu; ++s) {
          const bool last = l == 0 && s + 1 == mg.nu;
          if (work) {
            const double v = sweep(l, last);
            if (last) rz = v;
          }
          if (!last) {
            grid.sync();
            trace(10 * l + 6);
          }
        }
      }
    }
    const double bs = block_sum<kMgBlock>(rz);
    if (threadIdx.x == 0 && work) part_rz[vb] = bs;
    grid.sync();
    trace(7);
  }
};

// CG scalars as in the Jacobi solve: [0] rz, [3] rr (on exit the true
// residual's), [6] ||b||^2, [7] converged at the start, [8] iterations, [9]
// (rel_tol ||b||)^2, all written here, as is z = M r for the initial residual.
//
// K solves share the launch: block b works for solve b / grid on its own
// grid of `grid` blocks (local block b % grid), so each solve runs as it
// would alone.  Every block follows every solve's residual norm (each
// computes the same fixed-order sums), so all blocks agree on when the
// launch ends; a block whose solve has finished takes only the barriers.
// b_ff[n] and (b_ff - A x)[n] of the eliminated system: the free rows'
// right side with the Dirichlet neighbours' values folded in, and its
// residual (zero on Dirichlet rows).  x holds the Dirichlet values on
// Dirichlet nodes.  The folded_rhs / stencil_apply terms in their order.
__device__ __forceinline__ void folded_residual(const MgSystem &Y, const Grid3 &g, const double *x, int n,
                                                double &bf, double &rn) {
  if (Y.dirichlet[n]) {
    bf = rn = 0.0;
    return;
  }
  int i, j, k;
  node_ijk(n, g, i, j, k);
  const CoefRow a{Y.mg.L[0].st + n, g.px * g.py * g.pz};
  double acc = a[6] * x[n], fold = 0.0;
  const int nb[6] = {i > 0 ? n - g.pz : -1, i + 1 < g.px ? n + g.pz : -1, j > 0 ? n - g.px * g.pz : -1,
                     j + 1 < g.py ? n + g.px * g.pz : -1, k > 0 ? n - 1 : -1, k + 1 < g.pz ? n + 1 : -1};
#pragma unroll
  for (int t = 0; t < 6; ++t) {
    const int m = nb[t];
    if (m < 0 || a[t] == 0.0) continue;
    if (Y.dirichlet[m]) fold += a[t] * x[m];
    else acc += a[t] * x[m];
  }
  bf = Y.rhs[n] - fold;
  rn = bf - acc;
}

template <int K>
struct MgGroup {
  MgSystem s[K];
  int grid;
};

template <int K>
__device__ __forceinline__ void cg_mg_body(const MgGroup<K> &G) {
  cg::grid_group grid = cg::this_grid();
  const int nblk = G.grid;
  const int me = K == 1 ? 0 : (int)blockIdx.x / nblk;
  const int vb = (int)blockIdx.x - me * nblk;
  const MgSystem &Y = G.s[me];
  const Grid3 g{Y.px, Y.py, Y.pz};
  const int nodes = g.px * g.py * g.pz;
  const double *st7 = Y.mg.L[0].st;  // coefficient-major copy of the CG's 7-point stencil
  const uint8_t *dirichlet = Y.dirichlet;
  double *x = Y.x, *r = Y.r, *q = Y.q;
  double *part_pq = Y.part, *part_rz = Y.part + nblk, *part_rr = Y.part + 2 * nblk;
  Solve S{Y.mg, st7, g, vb * kMgBlock + (int)threadIdx.x, nblk * kMgBlock, 0u, r};
  // the CG update computes level 0's residual of the next V-cycle's first
  // sweep (one smoothing sweep: nothing runs between the two), reading the
  // neighbours' old residuals; so r alternates between two buffers
  const bool fuse_r0 = Y.mg.levels > 1 && Y.mg.nu == 1;
  const MgDevLevel &L0 = Y.mg.L[0];
  // set-up: the Dirichlet values into x, then r = b_ff - A x (x: the
  // previous potential, a warm start) and the partials of ||b_ff||^2, ||r||^2
  for (int n = S.tid; n < nodes; n += S.stride)
    if (dirichlet[n]) x[n] = Y.rhs[n];
  grid.sync();
  {
    double bb = 0.0, r2 = 0.0;
    for (int n = S.tid; n < nodes; n += S.stride) {
      double bf, rn;
      folded_residual(Y, g, x, n, bf, rn);
      r[n] = rn;
      bb += bf * bf;
      r2 += rn * rn;
    }
    const double s1 = block_sum<kMgBlock>(bb), s2 = block_sum<kMgBlock>(r2);
    if (threadIdx.x == 0) {
      part_pq[vb] = s1;
      part_rr[vb] = s2;
    }
  }
  grid.sync();
  bool done[K];
  int it[K];
  double tol2[K];
  bool any = false;
  double bnorm2 = 0.0, rr = 0.0, rz = 0.0, beta = 0.0;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const double b2 = sum_partials<kMgBlock>(G.s[k].part, nblk);
    const double r2 = sum_partials<kMgBlock>(G.s[k].part + 2 * nblk, nblk);
    tol2[k] = G.s[k].rel_tol2 * b2;
    done[k] = r2 <= tol2[k];  // converged already when the warm start meets the tolerance
    it[k] = 0;
    any = any || !done[k];
    if (k == me) {
      bnorm2 = b2;
      rr = r2;
    }
  }
  if (vb == 0 && threadIdx.x == 0) {
    Y.sc[6] = bnorm2;
    Y.sc[7] = done[me] ? 1.0 : 0.0;
    Y.sc[9] = tol2[me];
  }
  trace(0);
  if (any) {
    const bool work = !done[me];
    if (Y.mg.levels > 1) {
      if (work)
        for (int n = S.tid; n < nodes; n += S.stride) S.first(0, n, r[n]);
      grid.sync();
    }
    S.vcycle(grid, part_rz, vb, work, false);
    if (work) rz = sum_partials<kMgBlock>(part_rz, nblk);
  }
  const double *pin = Y.p0;
  double *pout = Y.p1;
  for (;;) {
    bool act[K];
    any = false;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      act[k] = !done[k] && it[k] < G.s[k].max_iter;
      any = any || act[k];
    }
    if (!any) break;
    const bool work = act[me];
    const double *z = S.X(0);
    double v = 0.0;
    if (work) {
      const int first = it[me] == 0;
      for (int n = S.tid; n < nodes; n += S.stride) {
        if (dirichlet[n]) {
          q[n] = 0.0;
          pout[n] = 0.0;
          continue;
        }
        // z and p vanish on Dirichlet nodes, so neighbours need no mask
        int i, j, k;
        node_ijk(n, g, i, j, k);
        const CoefRow a{st7 + n, nodes};
        // (pin is not read in the first iteration: it holds no p yet)
        auto P = [&](int m) { return first ? z[m] : z[m] + beta * pin[m]; };
        const double pn = P(n);
        pout[n] = pn;
        double acc = a[6] * pn;
        if (i > 0) acc += a[0] * P(n - g.pz);
        if (i + 1 < g.px) acc += a[1] * P(n + g.pz);
        if (j > 0) acc += a[2] * P(n - g.px * g.pz);
        if (j + 1 < g.py) acc += a[3] * P(n + g.px * g.pz);
        if (k > 0) acc += a[4] * P(n - 1);
        if (k + 1 < g.pz) acc += a[5] * P(n + 1);
        q[n] = acc;
        v += pn * acc;
      }
    }
    const double bs = block_sum<kMgBlock>(v);
    if (threadIdx.x == 0 && work) part_pq[vb] = bs;
    grid.sync();
    trace(100);
    double a2 = 0.0;
    if (work && fuse_r0) {
      const double alpha = rz / sum_partials<kMgBlock>(part_pq, nblk);
      const double *rin = S.b0;
      double *rout = rin == r ? Y.r1 : r;
      double *x0 = S.X(0);
      // first-sweep value of node m from its updated residual, as first(0)
      auto first0 = [&](int m) { return dirichlet[m] ? 0.0 : L0.fscale[m] * (rin[m] - alpha * q[m]); };
      const int sx = g.pz, sy = g.px * g.pz;
      for (int n = S.tid; n < nodes; n += S.stride) {
        double rn = rin[n];
        if (!dirichlet[n]) {
          x[n] += alpha * pout[n];
          rn = rin[n] - alpha * q[n];
          a2 += rn * rn;
        }
        rout[n] = rn;
        const double f = dirichlet[n] ? 0.0 : L0.fscale[n] * rn;
        x0[n] = f;
        // level 0's residual of the first sweep (apply7's terms and order;
        // an off-grid neighbour has a zero coefficient and is clamped)
        int i, j, k;
        node_ijk(n, g, i, j, k);
        const CoefRow a{st7 + n, nodes};
        double acc = a[6] * f;
        acc += a[0] * first0(i > 0 ? n - sx : n);
        acc += a[1] * first0(i + 1 < g.px ? n + sx : n);
        acc += a[2] * first0(j > 0 ? n - sy : n);
        acc += a[3] * first0(j + 1 < g.py ? n + sy : n);
        acc += a[4] * first0(k > 0 ? n - 1 : n);
        acc += a[5] * first0(k + 1 < g.pz ? n + 1 : n);
        const double v = rn - acc;
        L0.r[n] = L0.dir[n] ? 0.0 : v;
      }
      S.b0 = rout;
    } else if (work) {
      const double alpha = rz / sum_partials<kMgBlock>(part_pq, nblk);
      for (int n = S.tid; n < nodes; n += S.stride) {
        if (dirichlet[n]) {
          if (Y.mg.levels > 1) S.X(0)[n] = 0.0;
          continue;
        }
        x[n] += alpha * pout[n];
        const double rn = r[n] - alpha * q[n];
        r[n] = rn;
        a2 += rn * rn;
        if (Y.mg.levels > 1) S.first(0, n, rn);
      }
    }
    const double b2 = block_sum<kMgBlock>(a2);
    if (threadIdx.x == 0 && work) part_rr[vb] = b2;
    grid.sync();
    trace(101);
    // every solve's |r|^2, each in its own order
    bool more = false;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (!act[k]) continue;
      const double rk = sum_partials<kMgBlock>(G.s[k].part + 2 * nblk, nblk);
      if (k == me) rr = rk;
      ++it[k];
      done[k] = rk <= tol2[k];
      more = more || !done[k];
    }
    if (!more) break;
    const bool cycle = work && !done[me];
    S.vcycle(grid, part_rz, vb, cycle, fuse_r0);
    if (cycle) {
      const double rz_new = sum_partials<kMgBlock>(part_rz, nblk);
      beta = rz_new / rz;
      rz = rz_new;
      const double *t = pout;
      pout = const_cast<double *>(pin);
      pin = t;
    }
  }
  // the true residual of the final iterate (the recurrence's drifts from
  // it), and the solve's statistics.  The barrier: every block has read the
  // partials the loop ended on (the last update of x is behind one too).
  grid.sync();
  {
    double r2 = 0.0;
    for (int n = S.tid; n < nodes; n += S.stride) {
      double bf, rn;
      folded_residual(Y, g, x, n, bf, rn);
      r[n] = rn;
      r2 += rn * rn;
    }
    const double s2 = block_sum<kMgBlock>(r2);
    if (threadIdx.x == 0) part_rr[vb] = s2;
  }
  grid.sync();
  rr = sum_partials<kMgBlock>(part_rr, nblk);
  if (vb == 0 && threadIdx.x == 0) {
    Y.sc[0] = rz;
    Y.sc[3] = rr;
    Y.sc[8] = it[me];
    if (Y.stats) {
      const double bnorm = sqrt(bnorm2) > 0 ? sqrt(bnorm2) : 1.0;
      Y.stats[0] += 1.0;
      Y.stats[1] += it[me];
      Y.stats[2] = fmax(Y.stats[2], sqrt(rr) / bnorm);
    }
  }
}

// Preferred shared-memory carveout of the solve kernels, in per cent (-1:
// the driver's choice).  An SM's carveout is fixed while blocks run on it;
// with the driver's choice (the solve's blocks need 2 KB) a batched flight
// block (about 56 KB for a batch of 64) cannot join an SM running a solve,
// and 50 lets it.  Off by default: measured on the FinFET, 50 made the solve
// 9 % slower (less L1) for a batch overlap gain within the noise.
#ifndef MCB200_SOLVE_CARVEOUT
#define MCB200_SOLVE_CARVEOUT -1
#endif
// At most 64 registers a thread: a solve's block (512 threads) and one
// 256-thread block of the flight kernels fit in an SM's registers together
// (a solve can run beside a flight), and two blocks of the pair kernel fit alone.
// (Measured on the FinFET: the cap costs the solo solve about 2 %; without
// it the compiler's choice was slower still.)
__global__ void __launch_bounds__(kMgBlock, 1024 / kMgBlock) cg_mg_persistent(const __grid_constant__ MgGroup<1> G) {
  cg_mg_body<1>(G);
}
__global__ void __launch_bounds__(kMgBlock, 1024 / kMgBlock) cg_mg_pair(const __grid_constant__ MgGroup<2> G) {
  cg_mg_body<2>(G);
}

template <typename T>
T *upload(const std::vector<T> &v, std::vector<void *> &owned) {
  if (v.empty()) return nullptr;
  void *p = nullptr;
  if (cudaMalloc(&p, v.size() * sizeof(T)) != cudaSuccess) throw std::runtime_error("multigrid: cudaMalloc failed");
  owned.push_back(p);
  if (cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
    throw std::runtime_error("multigrid: upload failed");
  return static_cast<T *>(p);
}
double *scratch(size_t n, std::vector<void *> &owned) {
  void *p = nullptr;
  if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(double)) != cudaSuccess)
    throw std::runtime_error("multigrid: cudaMalloc failed");
  owned.push_back(p);
  cudaMemset(p, 0, std::max<size_t>(n, 1) * sizeof(double));
  return static_cast<double *>(p);
}

}  // namespace

MgDevice mg_upload(const MgHierarchy &h, const std::vector<double> &stencil7, std::vector<void *> &owned) {
  MgDevice d;
  d.levels = (int)h.levels.size();
  if (d.levels < 1 || d.levels > kMgMaxLevels) throw std::runtime_error("multigrid: bad level count");
  for (int l = 0; l < d.levels; ++l) {
    const MgLevel &s = h.levels[l];
    MgDevLevel &L = d.L[l];
    L.px = s.px;
    L.py = s.py;
    L.pz = s.pz;
    L.n = s.nodes();
    L.omega = s.omega;
    // stencils coefficient-major: level 0 the CG's 7-point one, else the 27-point Galerkin one
    const std::vector<double> &src = l == 0 ? stencil7 : s.st;
    const int w = l == 0 ? 7 : 27;
    if (src.size() != (size_t)L.n * w) throw std::runtime_error("multigrid: stencil size");
    std::vector<double> cm(src.size());
    for (int n = 0; n < L.n; ++n)
      for (int t = 0; t < w; ++t) cm[(size_t)t * L.n + n] = src[(size_t)n * w + t];
    L.st = upload(cm, owned);
    L.dinv = upload(s.dinv, owned);
    L.dir = upload(s.dir, owned);
    if (l > 0) {
      L.b = scratch(L.n, owned);
      L.xa = scratch(L.n, owned);
    }
    L.xb = scratch(L.n, owned);
    L.r = scratch(L.n, owned);
    if (l == 0) {
      std::vector<double> fs(L.n);
      for (int n = 0; n < L.n; ++n) fs[n] = s.dir[n] ? s.dinv[n] : s.omega * s.dinv[n];
      L.fscale = upload(fs, owned);
    }
    if (l + 1 < d.levels) {
      const MgAxis *ax[3] = {&s.ax, &s.ay, &s.az};
      const std::vector<int> *kp[3] = {&s.kx, &s.ky, &s.kz};
      for (int a = 0; a < 3; ++a) {
        const size_t m = ax[a]->c0.size();
        std::vector<int2> cm(m);
        std::vector<double2> wm(m);
        for (size_t i = 0; i < m; ++i) {
          cm[i] = make_int2(ax[a]->c0[i], ax[a]->c1[i]);
          wm[i] = make_double2(ax[a]->w0[i], ax[a]->w1[i]);
        }
        L.cmap[a] = upload(cm, owned);
        L.wmap[a] = upload(wm, owned);
        L.keep[a] = upload(*kp[a], owned);
        L.rtap[a] = upload(a == 0 ? s.rx : a == 1 ? s.ry : s.rz, owned);
      }
    }
  }
  d.coarse_inv = upload(h.coarse_inv, owned);
  return d;
}

#ifdef MCB200_MG_TRACE
extern "C" int mcb200_mg_trace_read(unsigned long long *out, int max_entries) {
  int n = 0;
  cudaMemcpyFromSymbol(&n, g_trace_n, sizeof(int));
  n = std::min(n, max_entries);
  cudaMemcpyFromSymbol(out, g_trace, 2 * n * sizeof(unsigned long long));
  const int zero = 0;
  cudaMemcpyToSymbol(g_trace_n, &zero, sizeof(int));
  return n;
}
#endif

// The carveout preference (MCB200_SOLVE_CARVEOUT), once per device.
static void configure_solve_kernels(int dev) {
  static unsigned long long done = 0;
  if (dev < 0 || dev >= 64 || ((done >> dev) & 1ull)) return;
  if (MCB200_SOLVE_CARVEOUT < 0 ||
      (cudaFuncSetAttribute(cg_mg_persistent, cudaFuncAttributePreferredSharedMemoryCarveout, MCB200_SOLVE_CARVEOUT) ==
           cudaSuccess &&
       cudaFuncSetAttribute(cg_mg_pair, cudaFuncAttributePreferredSharedMemoryCarveout, MCB200_SOLVE_CARVEOUT) ==
           cudaSuccess))
    done |= 1ull << dev;
  else
    cudaGetLastError();  // a hint only: the solves run without it
}

static int co_resident(const void *kernel) {
  int dev = 0, sms = 0, per_sm = 0, coop = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  configure_solve_kernels(dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
  if (!coop || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kMgBlock, 0) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return per_sm * sms;
}

int cg_mg_max_grid() { return co_resident((const void *)cg_mg_persistent); }

int cg_mg_blocks_per_sm() { return MCB200_MG_BLOCKS_PER_SM; }

bool cg_mg_pair_fits(int grid) { return grid > 0 && 2 * grid <= co_resident((const void *)cg_mg_pair); }

cudaError_t launch_cg_mg(const MgSystem &y, int grid, cudaStream_t s) {
  MgGroup<1> G;
  G.s[0] = y;
  G.grid = grid;
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) configure_solve_kernels(dev);
  void *args[] = {&G};
  return cudaLaunchCooperativeKernel((const void *)cg_mg_persistent, grid, kMgBlock, args, 0, s);
}

cudaError_t launch_cg_mg_pair(const MgSystem a[2], int grid, cudaStream_t s) {
  if (a[0].mg.levels != a[1].mg.levels || a[0].mg.nu != a[1].mg.nu || !cg_mg_pair_fits(grid))
    return cudaErrorInvalidValue;
  MgGroup<2> G;
  G.s[0] = a[0];
  G.s[1] = a[1];
  G.grid = grid;
  void *args[] = {&G};
  return cudaLaunchCooperativeKernel((const void *)cg_mg_pair, 2 * grid, kMgBlock, args, 0, s);
}

}  // namespace mcb200
