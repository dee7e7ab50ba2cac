// deck.h -- the reference's input decks, read on the host: input.txt
// (key = value), lgrid.txt (node coordinates) and ldg.txt (the device
// script), applied to per-cell arrays exactly as the reference's
// initialisation does (getInputData, read_grid_file, read_device_file,
// init_by_user_input, SetMRCube / SetMRPlane; src/mcmodel.cpp:3824-4693,
// src/set_user_defined_data.cpp), plus the derived cell data of
// init_cell_data, init_surface_roughness and compute_par_num.
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include "fullband_tables.h"

namespace mcb200 {

struct DeckError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// Material codes, include/Constant_GlobalVariable_MathFunction.h:165-175.
constexpr int kMatVacuum = 1, kMatOxide = 2, kMatSilicon = 3, kMatIgzo = 6;
constexpr int kMaxContactPlanes = 10;  // MNContactPlane

struct DeckContact {
  int nplanes = 0;
  double phims_v = 0, vapp_v = 0;     // volts, as written
  int plane[kMaxContactPlanes][6];    // node index ranges i0 i1 j0 j1 k0 k1
};

struct Deck {
  // ---- input.txt (getInputData, init_phpysical_parameter)
  std::string input_path, base_dir, grid_file, device_file, output_dir, restart_file;
  int total_step = 100000, electron_number = 100000, hole_number = 100000;
  int stat_step = 5000, stat_heat_step = 5000, heat_steps = 20000, mr_step = 10, restart_step = 0;
  double temperature = 300.0, dt_s = 1e-16;
  bool flag_multiple_refresh = false, flag_compute_potential = true, flag_compute_heat = false;
  bool flag_surface_scatter = true, flag_surface_roughness = true, flag_surface_phonon = true;
  bool flag_surface_impurity = false, flag_restart = false, flag_nonlinear_poisson = false;
  bool flag_quantum_correction = false;
  int quantum_start_step = 20;
  // ep_parm (keyword 15): window ratio and theta (nm) per axis, barrier Eb (V)
  double qc_ratio[3] = {0, 0, 0}, qc_theta_nm[3] = {0, 0, 0}, qc_eb_v = 0;
  // ---- lgrid.txt: node coordinates in metres (micrometres x 1e-6 as read)
  std::vector<double> lx_m, ly_m, lz_m;
  int nx = 0, ny = 0, nz = 0;
  // ---- ldg.txt applied to the cells, index (j * nx + i) * nz + k
  std::vector<int> material, desired_e, desired_h, attached_contact, scatter_type, in_surf, quantum_region;
  std::vector<int> motion;  // [cells][6]
  std::vector<double> donor_m3, acceptor_m3;
  int default_e = 0, default_h = 0;
  std::vector<DeckContact> contacts;
  int num_surfaces = 0;
  int surface_type[30] = {0}, surface_dir[30] = {0};
  double surface_pos_nm[30] = {0};

  // Parse input.txt and the grid / device files it names (relative to the
  // directory of input.txt).  Throws DeckError.
  static Deck load(const std::string &input_path);
  int cells() const { return nx * ny * nz; }
  int cell(int i, int j, int k) const { return (j * nx + i) * nz + k; }
};

// The deck in the reference's normalised units at the tables' temperature.
struct DeckScaled {
  std::vector<double> lx, ly, lz, dx, dy, dz;  // scaling(), src/mcmodel.cpp:4125-4166
  std::vector<double> donor, acceptor, volume, da;
  std::vector<double> init_e_charge, init_h_charge;  // init_cell_data, :3187-3270
  double sum_e = 0, sum_h = 0;
  std::vector<int> nearest_surf, eeff_dir;  // init_surface_roughness, :3155-3185
  double surface_pos[30] = {0};
  std::vector<int> electron_num, hole_num;  // compute_par_num, src/particle_init.cpp:17-74
  std::vector<int> desired_e, desired_h;    // raised by compute_par_num
  // Flag_restart: per-cell |q| sums of the restart file (its counts replace electron_num / hole_num)
  std::vector<double> restart_e_charge, restart_h_charge;
  std::vector<double> vapp, phims;          // per contact, / pot0
  double dt = 0;                            // / time0
  double qc_theta[3] = {0, 0, 0}, qc_eb = 0;  // ep_parm: theta / (1e9 spr0), Eb / pot0 (:4549-4556)

  static DeckScaled build(const Deck &d, const Units &u, double ni);
};

}  // namespace mcb200
