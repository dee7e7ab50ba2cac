// quantum_kernels.cu -- the effective potential of the quantum region
// (quantum_setup.h; MeshQuantities::effective_potential / quantumPotential,
// src/mcmodel.cpp:2337-2403).
#include "quantum_setup.h"

namespace mcb200 {

namespace {

__global__ void copy_potential_kernel(int nodes, const double *pot, double *out) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n < nodes) out[n] = pot[n];
}

// One thread per quantum node; the window is summed in the reference's
// order (x outer, z inner) and the product of the three erf differences in
// its association ((V + Eb) * dz) * dy) * dx.  Every term reads `pot`, never
// `out`, so no node sees another's corrected value.
__global__ void effective_potential_kernel(QuantumDevice q, const double *pot, double *out) {
  const size_t nodes = (size_t)q.px * q.py * q.pz;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < q.n_list; t += gridDim.x * blockDim.x) {
    const int n = q.list[t];
    const int pk = n % q.pz, r = n / q.pz, pi = r % q.px, pj = r / q.px;
    const int2 wx = q.window[pi], wy = q.window[q.px + pj], wz = q.window[q.px + q.py + pk];
    const double qx = q.qcl[pi], qy = q.qcl[q.px + pj], qz = q.qcl[q.px + q.py + pk];
    double ret = 0.0;
    for (int i = wx.x; i <= wx.y; ++i)
      for (int j = wy.x; j <= wy.y; ++j)
        for (int k = wz.x; k <= wz.y; ++k) {
          const size_t m = ((size_t)j * q.px + i) * q.pz + k;
          if (!q.inside[m]) continue;
          const double v = pot[m] + q.eb[m];
          const double x1 = q.range[m] - qx, x2 = q.range[nodes + m] - qx;
          const double y1 = q.range[2 * nodes + m] - qy, y2 = q.range[3 * nodes + m] - qy;
          const double z1 = q.range[4 * nodes + m] - qz, z2 = q.range[5 * nodes + m] - qz;
          ret += v * (erf(z2) - erf(z1)) * (erf(y2) - erf(y1)) * (erf(x2) - erf(x1));
        }
    out[n] = ret * 0.125;
  }
}

}  // namespace

void launch_effective_potential(const QuantumDevice &q, const double *pot, double *out, cudaStream_t s) {
  const int nodes = q.px * q.py * q.pz;
  if (nodes <= 0) return;
  copy_potential_kernel<<<(nodes + 255) / 256, 256, 0, s>>>(nodes, pot, out);
  if (q.n_list > 0) effective_potential_kernel<<<(q.n_list + 127) / 128, 128, 0, s>>>(q, pot, out);
}

}  // namespace mcb200
