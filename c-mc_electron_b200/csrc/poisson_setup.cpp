// poisson_setup.cpp -- see poisson_setup.h.  Compiled with -ffp-contract=off.
#include "poisson_setup.h"

#include <cmath>
#include <stdexcept>

namespace mcb200 {

namespace {
constexpr int kVacuum = 1;
constexpr int kSilicon = 3;
}  // namespace

PoissonSetup PoissonSetup::build(int nx, int ny, int nz, const double *dx, const double *dy, const double *dz,
                                 const int32_t *material, const double *donor, const double *acceptor, double ni,
                                 const double *eps, const std::vector<ContactPlane> &planes,
                                 const std::vector<double> &vapp, const std::vector<double> &phims) {
  PoissonSetup s;
  s.nx = nx;
  s.ny = ny;
  s.nz = nz;
  const int cells = nx * ny * nz, nodes = s.nodes();
  s.cvol.assign(cells, 0.0);
  s.pvol.assign(nodes, 0.0);
  s.pdop.assign(nodes, 0.0);
  s.vadd.assign(nodes, 0.0);
  s.stencil.assign((size_t)nodes * 7, 0.0);
  s.dirichlet.assign(nodes, 0);
  s.bc_vapp.assign(nodes, 0.0);
  s.contact_of.assign(nodes, -1);
  s.bc_phims.assign(nodes, 0.0);

  // init_cell_data, src/mcmodel.cpp:3213-3218: cell volumes
  for (int i = 0; i < nx; ++i)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j) s.cvol[s.cell(i, j, k)] = dx[i] * dy[j] * dz[k];

  // init_point_data, :3294-3330: each silicon cell gives an eighth of its
  // volume and doping to each of its nodes (same node order as the reference)
  for (int i = 0; i < nx; ++i)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j) {
        const int c = s.cell(i, j, k);
        if (material[c] != kSilicon) continue;
        const double vol_tmp = s.cvol[c] * 0.125;
        const double da_tmp = vol_tmp * (donor[c] - acceptor[c]);
        const int lo[4] = {s.node(i + 1, j, k), s.node(i, j, k), s.node(i + 1, j, k + 1), s.node(i, j, k + 1)};
        const int hi[4] = {s.node(i + 1, j + 1, k), s.node(i, j + 1, k), s.node(i + 1, j + 1, k + 1),
                           s.node(i, j + 1, k + 1)};
        for (int q = 0; q < 4; ++q) s.pdop[lo[q]] += da_tmp;
        for (int q = 0; q < 4; ++q) s.pdop[hi[q]] += da_tmp;
        for (int q = 0; q < 4; ++q) s.pvol[lo[q]] += vol_tmp;
        for (int q = 0; q < 4; ++q) s.pvol[hi[q]] += vol_tmp;
      }
  // :3335-3355: built-in potential of the net doping
  for (int i = 0; i <= nx; ++i)
    for (int k = 0; k <= nz; ++k)
      for (int j = 0; j <= ny; ++j) {
        const int p = s.node(i, j, k);
        const double ndop = std::fabs(s.pvol[p]) > 1e-16 ? s.pdop[p] / s.pvol[p] : 0;
        const double alfa = ndop / (ni * 2.0);
        if (alfa > 0.0)
          s.vadd[p] = std::log(alfa + std::sqrt(1.0 + alfa * alfa));
        else if (alfa < 0)
          s.vadd[p] = -std::log(std::sqrt(1.0 + alfa * alfa) - alfa);
        else
          s.vadd[p] = 0;
      }
  // :3356-3363: the first and last y node planes copy their inner neighbours
  for (int i = 0; i <= nx; ++i)
    for (int k = 0; k <= nz; ++k) s.vadd[s.node(i, ny, k)] = s.vadd[s.node(i, ny - 1, k)];
  for (int i = 0; i <= nx; ++i)
    for (int k = 0; k <= nz; ++k) s.vadd[s.node(i, 0, k)] = s.vadd[s.node(i, 1, k)];

  // init_matrix, :4695-4869: FV stencil accumulated cell by cell
  auto add = [&](int p, int slot, double v) { s.stencil[(size_t)p * 7 + slot] += v; };
  for (int i = 0; i < nx; ++i)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j) {
        const int m = material[s.cell(i, j, k)];
        if (m == kVacuum) continue;
        if (m < 0 || m > 5) throw std::runtime_error("material index out of range");
        const double eps0 = eps[m];
        const double AA = -0.25 * eps0 * dx[i] * dy[j] / dz[k];
        const double BB = -0.25 * eps0 * dx[i] * dz[k] / dy[j];
        const double CC = -0.25 * eps0 * dz[k] * dy[j] / dx[i];
        const double DD = -AA - BB - CC;
        // {node, z slot, y slot, x slot}
        const int low[4][4] = {{s.node(i, j, k), 5, 3, 1}, {s.node(i, j, k + 1), 4, 3, 1},
                               {s.node(i + 1, j, k), 5, 3, 0}, {s.node(i + 1, j, k + 1), 4, 3, 0}};
        const int high[4][4] = {{s.node(i, j + 1, k), 5, 2, 1}, {s.node(i, j + 1, k + 1), 4, 2, 1},
                                {s.node(i + 1, j + 1, k), 5, 2, 0}, {s.node(i + 1, j + 1, k + 1), 4, 2, 0}};
        for (const auto *set : {low, high})
          for (int q = 0; q < 4; ++q) {
            add(set[q][0], set[q][1], AA);
            add(set[q][0], set[q][2], BB);
            add(set[q][0], set[q][3], CC);
            add(set[q][0], 6, DD);
          }
      }
  for (int p = 0; p < nodes; ++p) {
    bool any = false;
    for (int q = 0; q < 7; ++q) any = any || s.stencil[(size_t)p * 7 + q] != 0;
    if (!any) s.stencil[(size_t)p * 7 + 6] = 1;
  }
  for (const ContactPlane &pl : planes) {
    if (pl.contact < 0 || pl.contact >= (int)vapp.size()) throw std::runtime_error("contact plane without contact");
    for (int i = pl.i0; i <= pl.i1; ++i)
      for (int k = pl.k0; k <= pl.k1; ++k)
        for (int j = pl.j0; j <= pl.j1; ++j) {
          if (i < 0 || i > nx || j < 0 || j > ny || k < 0 || k > nz) throw std::runtime_error("contact plane off the mesh");
          const int p = s.node(i, j, k);
          for (int q = 0; q < 7; ++q) s.stencil[(size_t)p * 7 + q] = 0;
          s.stencil[(size_t)p * 7 + 6] = 1;
          s.dirichlet[p] = 1;
          s.bc_vapp[p] = vapp[pl.contact];
          s.bc_phims[p] = phims[pl.contact];
          s.contact_of[p] = (int8_t)pl.contact;
        }
  }
  return s;
}

}  // namespace mcb200
