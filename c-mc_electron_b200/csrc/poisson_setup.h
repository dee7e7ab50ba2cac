// poisson_setup.h -- host-side assembly of the device description used by
// deposition and the Poisson solve: cell and node volumes, node doping, the
// built-in potential vadd, the 7-point finite-volume stencil with Dirichlet
// contact rows, and the contact potentials.
//
// Restates MeshQuantities::init_cell_data (src/mcmodel.cpp:3187-3270),
// init_point_data (:3272-3390) and init_matrix (:4695-4869) for one rank,
// keeping their summation order so the stencil and node data are
// bit-identical to the reference's.
#pragma once

#include <cstdint>
#include <vector>

namespace mcb200 {

struct ContactPlane {
  int contact;                 // 0-based contact index
  int i0, i1, j0, j1, k0, k1;  // inclusive node ranges
};

struct PoissonSetup {
  int nx = 0, ny = 0, nz = 0;  // cells
  std::vector<double> cvol;     // [cells]
  std::vector<double> pvol;     // [nodes] node control volume (silicon cells only)
  std::vector<double> pdop;     // [nodes] integrated doping (donor - acceptor), silicon cells only
  std::vector<double> vadd;     // [nodes] built-in potential asinh(N / 2 Ni)
  std::vector<double> stencil;  // [nodes][7]: -x, +x, -y, +y, -z, +z, diagonal
  std::vector<uint8_t> dirichlet;   // [nodes] contact rows
  std::vector<double> bc_vapp, bc_phims;  // [nodes] the contact's Vapp and PhiMS on Dirichlet rows
  std::vector<int8_t> contact_of;         // [nodes] the contact of a Dirichlet row, -1 elsewhere

  int nodes() const { return (nx + 1) * (ny + 1) * (nz + 1); }
  int node(int i, int j, int k) const { return (j * (nx + 1) + i) * (nz + 1) + k; }
  int cell(int i, int j, int k) const { return (j * nx + i) * nz + k; }

  // dx/dy/dz: cell widths (the reference's scaled dx/dy/dz); material per
  // cell (0 void, 1 vacuum, 2 oxide, 3 silicon); donor / acceptor per cell
  // (normalised); eps per material (6 entries); vapp / phims per contact.
  static PoissonSetup build(int nx, int ny, int nz, const double *dx, const double *dy, const double *dz,
                            const int32_t *material, const double *donor, const double *acceptor, double ni,
                            const double *eps, const std::vector<ContactPlane> &planes,
                            const std::vector<double> &vapp, const std::vector<double> &phims);
};

}  // namespace mcb200
