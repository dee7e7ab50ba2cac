// cell_kernels.cu -- per-cell kernels: surface scattering rates and
// MultipleRefresh.
//
//  * surface_rates: MeshQuantities::GetSurfRoughnessPhononScRate
//    (src/GetSurfRoughnessPhononScRate.cpp:4-70), one thread per cell, for
//    electrons and holes.  Inputs are the cell field (both carriers feel the
//    same field here), the screening density and the direction of the
//    nearest Si/SiO2 surface.
//  * multiple refresh: MeshQuantities::MultipleRefresh / gen_new_par_mr
//    (src/MultipleRefresh.cpp:9-143), one thread per cell.  The store is
//    sorted by cell; inside a cell the particles are taken in uid order
//    (the reference takes its list order).  Each (cell, carrier) draws from
//    its own stream (seed, cell, step, kRefreshSub + type).  Resampled
//    particles get fresh uids in (cell, type, draw) order.
#include "cell_kernels.h"
#include "pdl.cuh"

namespace mcb200 {

constexpr double kPiC = 3.141592653589793238462643e0;

__global__ void surface_rates_kernel(int cells, SurfaceRateParams q, const double *field, const double *rho,
                                     const int *eeff_dir, double *e_rough, double *e_phon, double *h_rough,
                                     double *h_phon) {
  pdl_wait();
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cells) return;
  const double Rho = rho[c];
  double Eeff = fabs(field[3 * (size_t)c + min(max(eeff_dir[c], 0), 2)]);
  if (Eeff < 1e-20) Eeff = 1e-20;
  // the per-cell powers, shared by both carrier types; the constant ones come from the host
  double e_third = 0, Pf = 0, Wcl = 0;
  if (q.phonon) {
    e_third = pow(Eeff, -1.0 / 3.0);
    Pf = q.pft * q.Tn + q.pfn * pow(Rho * q.conc0 / (1e17 * 1e6), q.npf) / q.Tn;
    Wcl = q.tn_nbmod * q.boltz * q.T0 / (Eeff * q.field0);
  }
  for (int t = 0; t < 2; ++t) {
    const double effmass = t == 0 ? 0.286 : 0.8;  // MASSeff, src/Constant_GlobalVariable_MathFunction.cpp:28
    double rough = 0, phon = 0;
    if (q.roughness) {
      const double a = q.delta * q.ail * Eeff * q.eps_si / (q.eps_si + q.eps_ox);
      rough = 2 * kPiC * effmass * (a * a);
    }
    if (q.phonon) {
      const double Wq = q.wq_c[t] * e_third;
      const double Wclq = (q.gama * Wcl + q.theta * Wq) / Pf;
      phon = effmass * q.em0 * q.boltz * q.T0 * q.xiph * q.xiph /
                 (q.hq0 * q.hq0 * q.hq0 * q.sirho * (9050.02 * 9050.02) * Wclq) / q.scrt0 +
             q.ec0 / (effmass * q.em0 * q.kpha * q.tn_224) / q.scrt0;
    }
    if (t == 0) { e_rough[c] = rough; e_phon[c] = phon; }
    else { h_rough[c] = rough; h_phon[c] = phon; }
  }
}

// ---------------------------------------------------------------------------
// MultipleRefresh.  Pass 1 (count): index each cell's particles in uid
// order (the cell is contiguous in the cell-sorted store), decide per carrier
// whether to resample and how many particles the cell will hold.  Pass 2 (emit): write the cell's
// new population at its scanned offset.
struct Decision {
  int keep;      // 1: keep the old population of this type
  int old_num;   // particles with |q| >= pckill
  double tot;    // their total charge
};

// The cell's particles [b, e) in uid order, as keys uid << 32 | index in
// order[b, e) (shell sort, Ciura's gaps): the refresh visits particles in
// uid order without moving the store.
__device__ void order_cell_by_uid(const uint32_t *uid, unsigned long long *order, int b, int e) {
  const int n = e - b;
  unsigned long long *a = order + b;
  for (int i = 0; i < n; ++i) a[i] = ((unsigned long long)uid[b + i] << 32) | (unsigned)(b + i);
  const int gaps[10] = {3937, 1750, 701, 301, 132, 57, 23, 10, 4, 1};
  for (int g : gaps) {
    if (g >= n) continue;
    for (int i = g; i < n; ++i) {
      const unsigned long long t = a[i];
      int j = i;
      while (j >= g && a[j - g] > t) {
        a[j] = a[j - g];
        j -= g;
      }
      a[j] = t;
    }
  }
}
__device__ __forceinline__ int nth(const unsigned long long *order, int k) { return (int)(order[k] & 0xffffffffull); }

// gen_new_par_mr's test (src/MultipleRefresh.cpp:18-33) for one carrier type.
template <typename R>
__device__ Decision decide(const DevParticlesT<R> &P, const unsigned long long *order, int b, int e, int type,
                           int new_num, const RefreshParams &r) {
  Decision d{1, 0, 0.0};
  double tmp = 0;
  for (int k = b; k < e; ++k) {
    const int i = nth(order, k);
    if (((P.meta[i] >> 8) & 255) != (uint32_t)type || fabs(P.charge[i]) < r.pckill) continue;
    d.old_num++;
    d.tot += P.charge[i];
    tmp += P.charge[i] * P.charge[i];
  }
  if (d.old_num == 0) return d;
  if (((d.old_num > new_num / r.rpar) && (d.old_num < new_num * r.rpar)) &&
      (tmp < (d.tot * d.tot * r.rsqr / d.old_num)))
    return d;
  d.keep = 0;
  return d;
}

template <typename R>
__global__ void refresh_count_kernel(DevParticlesT<R> P, const unsigned int *cell_end, const unsigned int *cell_count,
                                     int cells, const int *desired_e, const int *desired_h, RefreshParams r,
                                     unsigned long long *order, unsigned int *out_count, unsigned int *new_count) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cells) return;
  const int e = (int)cell_end[c], b = e - (int)cell_count[c];
  order_cell_by_uid(P.uid, order, b, e);
  unsigned int total = 0, fresh = 0;
  for (int t = 0; t < 2; ++t) {
    const int want = t == 0 ? desired_e[c] : desired_h[c];
    const Decision d = decide(P, order, b, e, t, want, r);
    if (d.keep) total += d.old_num;
    else {
      total += want;
      fresh += want;
    }
  }
  out_count[c] = total;
  new_count[c] = fresh;
}

template <typename R>
__global__ void refresh_emit_kernel(DevParticlesT<R> P, const unsigned int *cell_end, const unsigned int *cell_count,
                                    int cells, const int *desired_e, const int *desired_h, RefreshParams r,
                                    const unsigned long long *order, double *wsum, int *widx,
                                    const unsigned int *out_offset, const unsigned int *uid_offset,
                                    const unsigned int *uid0p, DevParticlesT<R> dst, unsigned long long *mr_gen) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cells) return;
  const int e = (int)cell_end[c], b = e - (int)cell_count[c];
  unsigned int o = out_offset[c];
  uint32_t uid = *uid0p + uid_offset[c];
  auto copy = [&](int from, unsigned int to) {
    dst.x[to] = P.x[from]; dst.y[to] = P.y[from]; dst.z[to] = P.z[from];
    dst.kx[to] = P.kx[from]; dst.ky[to] = P.ky[from]; dst.kz[to] = P.kz[from];
    dst.energy[to] = P.energy[from]; dst.charge[to] = P.charge[from];
    dst.cell[to] = P.cell[from]; dst.itet[to] = P.itet[from]; dst.meta[to] = P.meta[from] & 0xffffu;
    dst.uid[to] = P.uid[from];
  };
  int produced = 0;
  for (int t = 0; t < 2; ++t) {
    const int want = t == 0 ? desired_e[c] : desired_h[c];
    const Decision d = decide(P, order, b, e, t, want, r);
    if (d.keep) {
      for (int k = b; k < e; ++k) {
        const int i = nth(order, k);
        if (((P.meta[i] >> 8) & 255) == (uint32_t)t && fabs(P.charge[i]) >= r.pckill) copy(i, o++);
      }
      produced += d.old_num;
      continue;
    }
    // draw `want` particles with probability |q| / sum|q| (lower_bound on the
    // running sum, src/MultipleRefresh.cpp:35-44); the new charge is tot/want.
    // The running sums of |q| over this type's particles in uid order go to
    // wsum[b, b + m) once (m = d.old_num >= 1 here: an empty type is kept);
    // each draw then searches them.  The sums never decrease, so the first
    // one not below s is the one a scan would stop at.
    int m = 0;
    double w = 0;
    for (int k = b; k < e; ++k) {
      const int i = nth(order, k);
      if (((P.meta[i] >> 8) & 255) != (uint32_t)t || fabs(P.charge[i]) < r.pckill) continue;
      w += fabs(P.charge[i]);
      wsum[b + m] = w;
      widx[b + m] = i;
      ++m;
    }
    const double aver = d.tot / want;
    for (int q = 0; q < want; ++q) {
      const double s = mcb200_uniform(r.seed, (uint32_t)c, r.step, kRefreshSub + t, (uint32_t)q) * fabs(d.tot);
      int lo = 0, hi = m;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (wsum[b + mid] >= s) hi = mid;
        else lo = mid + 1;
      }
      // s above the last sum (rounding): the reference prints and skips; keep the count
      const int pick = widx[b + min(lo, m - 1)];
      copy(pick, o);
      dst.charge[o] = aver;
      dst.uid[o] = uid++;
      ++o;
    }
    produced += want;
  }
  atomicAdd(mr_gen, (unsigned long long)(long long)(produced - (e - b)));
}

void launch_surface_rates(int cells, const SurfaceRateParams &q, const double *field, const double *rho,
                          const int *eeff_dir, double *e_rough, double *e_phon, double *h_rough, double *h_phon,
                          cudaStream_t s) {
  launch_pdl(surface_rates_kernel, (cells + 255) / 256, 256, 0, s, cells, q, field, rho, eeff_dir, e_rough, e_phon,
             h_rough, h_phon);
}
template <typename R>
void launch_refresh_count(const DevParticlesT<R> &P, const unsigned int *cell_end, const unsigned int *cell_count,
                          int cells, const int *desired_e, const int *desired_h, const RefreshParams &r,
                          unsigned long long *order, unsigned int *out_count, unsigned int *new_count,
                          cudaStream_t s) {
  refresh_count_kernel<R><<<(cells + 127) / 128, 128, 0, s>>>(P, cell_end, cell_count, cells, desired_e, desired_h, r,
                                                           order, out_count, new_count);
}
template <typename R>
void launch_refresh_emit(const DevParticlesT<R> &P, const unsigned int *cell_end, const unsigned int *cell_count,
                         int cells, const int *desired_e, const int *desired_h, const RefreshParams &r,
                         const unsigned long long *order, double *wsum, int *widx, const unsigned int *out_offset,
                         const unsigned int *uid_offset, const unsigned int *uid0, const DevParticlesT<R> &dst,
                         unsigned long long *mr_gen, cudaStream_t s) {
  refresh_emit_kernel<R><<<(cells + 127) / 128, 128, 0, s>>>(P, cell_end, cell_count, cells, desired_e, desired_h, r,
                                                          order, wsum, widx, out_offset, uid_offset, uid0, dst,
                                                          mr_gen);
}

#define MCB200_INSTANTIATE(R)                                                                                 \
  template void launch_refresh_count<R>(const DevParticlesT<R> &, const unsigned int *, const unsigned int *, \
                                        int, const int *, const int *, const RefreshParams &,                 \
                                        unsigned long long *, unsigned int *, unsigned int *, cudaStream_t);  \
  template void launch_refresh_emit<R>(const DevParticlesT<R> &, const unsigned int *, const unsigned int *,  \
                                       int, const int *, const int *, const RefreshParams &,                 \
                                       const unsigned long long *, double *, int *, const unsigned int *,     \
                                       const unsigned int *, const unsigned int *, const DevParticlesT<R> &,  \
                                       unsigned long long *, cudaStream_t);
MCB200_INSTANTIATE(double)
MCB200_INSTANTIATE(float)
#undef MCB200_INSTANTIATE

}  // namespace mcb200
