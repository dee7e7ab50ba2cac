// quantum_setup.h -- the effective-potential quantum correction of the
// electron potential: host set-up (quantum_setup.cpp) and the GPU pass
// (quantum_kernels.cu).
//
// The reference smooths the Poisson potential (plus a barrier Eb on oxide
// nodes) over a Gaussian window at every node of the quantum region and
// gives electrons the field of the smoothed potential; holes keep the field
// of the plain potential (MeshQuantities::effective_potential /
// quantumPotential, src/mcmodel.cpp:2337-2403; set-up init_ep_range,
// init_p_mat, init_effective_potential, :2406-2664; applied in
// compute_field, :2240-2262).  At quantum node (pi, pj, pk):
//
//   V_eff = 1/8 sum over nodes n of the window with oxide or silicon,
//           (V[n] + Eb[n]) * prod over axes (erf(b2[n] - q[p]) - erf(b1[n] - q[p]))
//
// where b1 / b2 are the node's box edges (half way to its neighbours, or
// ratio * theta out where the neighbour is neither oxide nor silicon) and q
// the target's coordinate, all in units of sqrt(2) * theta per axis.
#pragma once

#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

namespace mcb200 {

// ep_parm (read_device_file keyword 15, src/mcmodel.cpp:4549-4556), in the
// normalised units: window half-widths in units of theta, theta, and the
// oxide barrier.
struct QuantumParams {
  double ratio[3] = {0, 0, 0};
  double theta[3] = {0, 0, 0};
  double eb = 0;
};

// Per-node data of the correction for a px x py x pz node grid (node (i, j, k)
// at (j * px + i) * pz + k).
struct QuantumHost {
  std::vector<uint8_t> inside;   // node of an oxide or silicon cell
  std::vector<double> eb;        // -Eb on oxide nodes that are not silicon, else 0
  std::vector<double> range;     // [6][nodes]: x1, x2, y1, y2, z1, z2
  std::vector<double> qcl;       // [px + py + pz]: node coordinate / (sqrt 2 theta), per axis
  std::vector<int> lower, upper; // [px + py + pz]: window of each node index, per axis
  std::vector<int> list;         // the quantum nodes
};

// init_effective_potential + init_p_mat + init_ep_range for one rank.
// Coordinates and widths normalised (mcb200_set_mesh); material and
// quantum_region per cell, index (j * nx + i) * nz + k.
QuantumHost quantum_setup(int nx, int ny, int nz, const double *lx, const double *ly, const double *lz,
                          const double *dx, const double *dy, const double *dz, const int32_t *material,
                          const int32_t *quantum_region, const QuantumParams &p);

// The same on the device.
struct QuantumDevice {
  int px = 0, py = 0, pz = 0, n_list = 0;
  const int *list = nullptr;
  const uint8_t *inside = nullptr;
  const double *eb = nullptr;
  const double *range = nullptr;
  const double *qcl = nullptr;
  const int2 *window = nullptr;  // (lower, upper) per axis index
};

// out = pot, with the effective potential at every quantum node (computed
// from pot, not from out).
void launch_effective_potential(const QuantumDevice &q, const double *pot, double *out, cudaStream_t s);

}  // namespace mcb200
