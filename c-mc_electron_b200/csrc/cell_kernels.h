// cell_kernels.h -- per-cell kernels (cell_kernels.cu): surface scattering
// rates and MultipleRefresh.
#pragma once

#include <cuda_runtime.h>

#include "device_state.cuh"
#include "mcb200_rng.h"

namespace mcb200 {

// `sub` word of the refresh streams: kRefreshSub + carrier type.
constexpr uint32_t kRefreshSub = 0x4d520000u;

// GetSurfRoughnessPhononScRate inputs: the SurfSc_* parameters
// (src/mcmodel.cpp:4107-4121) and the unit constants they are combined with.
struct SurfaceRateParams {
  double delta, ail, xiph, theta, gama, nbmod, npf, pft, pfn, kpha;
  int roughness, phonon;
  double eps_si, eps_ox, Tn, T0, boltz, field0, em0, ec0, hq0, conc0, sirho, scrt0;
  // derived on the host: Tn^nbmod, Tn^2.24 and, per carrier type,
  // (12 m* em0 field0 / ec0 / hq0^2)^(-1/3) (the field-independent factor of Wq)
  double tn_nbmod, tn_224, wq_c[2];
};

struct RefreshParams {
  uint64_t seed;
  uint32_t step;
  double rpar, rsqr, pckill;
};

void launch_surface_rates(int cells, const SurfaceRateParams &q, const double *field, const double *rho,
                          const int *eeff_dir, double *e_rough, double *e_phon, double *h_rough, double *h_phon,
                          cudaStream_t s);
template <typename R>
void launch_refresh_count(const DevParticlesT<R> &P, const unsigned int *cell_end, const unsigned int *cell_count,
                          int cells, const int *desired_e, const int *desired_h, const RefreshParams &r,
                          unsigned long long *order, unsigned int *out_count, unsigned int *new_count,
                          cudaStream_t s);
// order: one key per store slot, written by the count pass (each cell's
// particles in uid order) and read by the emit pass.  wsum / widx: one
// entry per store slot, the emit pass's running sums and their particles.
// uid0: device word holding the first new uid (the context's uid counter).
template <typename R>
void launch_refresh_emit(const DevParticlesT<R> &P, const unsigned int *cell_end, const unsigned int *cell_count,
                         int cells, const int *desired_e, const int *desired_h, const RefreshParams &r,
                         const unsigned long long *order, double *wsum, int *widx, const unsigned int *out_offset,
                         const unsigned int *uid_offset, const unsigned int *uid0, const DevParticlesT<R> &dst,
                         unsigned long long *mr_gen, cudaStream_t s);

}  // namespace mcb200
