// deck_api.cpp -- the C ABI of the deck reader (include/mcb200.h):
// load a deck, inspect it, normalise it with a context's units, and apply it
// to the context (mesh, cells, device, initial ensemble).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "deck.h"
#include "mcb200.h"

using namespace mcb200;

struct mcb200_deck {
  std::string error;
  bool loaded = false;
  Deck d;
  bool prepared = false;
  DeckScaled s;
};

namespace {

int deck_fail(mcb200_deck *k, int code, const std::string &msg) {
  if (k) k->error = msg;
  return code;
}

template <typename T>
int copy_out(const std::vector<T> &v, T *out, size_t n, size_t *needed) {
  if (needed) *needed = v.size();
  if (!out) return MCB200_OK;
  if (n < v.size()) return MCB200_ERR_CAPACITY;
  std::copy(v.begin(), v.end(), out);
  return MCB200_OK;
}

std::vector<int32_t> contact_planes(const Deck &d) {
  std::vector<int32_t> p;
  for (size_t c = 0; c < d.contacts.size(); ++c)
    for (int q = 0; q < d.contacts[c].nplanes; ++q) {
      p.push_back((int32_t)c);
      for (int e = 0; e < 6; ++e) p.push_back(d.contacts[c].plane[q][e]);
    }
  return p;
}

}  // namespace

extern "C" {

int mcb200_deck_load(const char *input_path, mcb200_deck **out) {
  if (!out || !input_path) return MCB200_ERR_ARG;
  mcb200_deck *k = new mcb200_deck;
  *out = k;
  try {
    k->d = Deck::load(input_path);
    k->loaded = true;
    return MCB200_OK;
  } catch (const std::exception &e) {
    return deck_fail(k, MCB200_ERR_IO, e.what());
  }
}

void mcb200_deck_free(mcb200_deck *deck) { delete deck; }

const char *mcb200_deck_error(const mcb200_deck *deck) { return deck ? deck->error.c_str() : "null deck"; }

int mcb200_deck_get_info(const mcb200_deck *k, mcb200_deck_info *info) {
  if (!k || !info) return MCB200_ERR_ARG;
  if (!k->loaded) return MCB200_ERR_STATE;
  const Deck &d = k->d;
  std::memset(info, 0, sizeof(*info));
  info->nx = d.nx; info->ny = d.ny; info->nz = d.nz;
  info->total_step = d.total_step;
  info->electron_number = d.electron_number;
  info->hole_number = d.hole_number;
  info->stat_step = d.stat_step;
  info->stat_heat_step = d.stat_heat_step;
  info->heat_steps = d.heat_steps;
  info->mr_step = d.mr_step;
  info->temperature = d.temperature;
  info->dt_s = d.dt_s;
  info->flag_multiple_refresh = d.flag_multiple_refresh;
  info->flag_compute_potential = d.flag_compute_potential;
  info->flag_compute_heat = d.flag_compute_heat;
  info->flag_surface_scatter = d.flag_surface_scatter;
  info->flag_surface_roughness = d.flag_surface_roughness;
  info->flag_surface_phonon = d.flag_surface_phonon;
  info->flag_surface_impurity = d.flag_surface_impurity;
  info->flag_restart = d.flag_restart;
  info->flag_quantum_correction = d.flag_quantum_correction;
  info->restart_step = d.restart_step;
  info->quantum_start_step = d.quantum_start_step;
  info->n_contacts = (int)d.contacts.size();
  int planes = 0;
  for (const auto &c : d.contacts) planes += c.nplanes;
  info->n_planes = planes;
  info->n_surfaces = d.num_surfaces;
  info->default_electrons = d.default_e;
  info->default_holes = d.default_h;
  std::strncpy(info->output_dir, d.output_dir.c_str(), sizeof(info->output_dir) - 1);
  info->prepared = k->prepared;
  info->dt = k->prepared ? k->s.dt : 0.0;
  return MCB200_OK;
}

int mcb200_deck_int_array(const mcb200_deck *k, const char *name, int32_t *out, size_t n, size_t *needed) {
  if (!k || !name) return MCB200_ERR_ARG;
  if (!k->loaded) return MCB200_ERR_STATE;
  const Deck &d = k->d;
  const std::string nm(name);
  const std::vector<int> *v = nullptr;
  std::vector<int> tmp;
  if (nm == "material") v = &d.material;
  else if (nm == "desired_electrons") v = &d.desired_e;
  else if (nm == "desired_holes") v = &d.desired_h;
  else if (nm == "attached_contact") v = &d.attached_contact;
  else if (nm == "scatter_type") v = &d.scatter_type;
  else if (nm == "in_surf_region") v = &d.in_surf;
  else if (nm == "quantum_region") v = &d.quantum_region;
  else if (nm == "motion_rule") v = &d.motion;
  else if (nm == "contact_planes") { tmp = contact_planes(d); v = &tmp; }
  else if (nm == "surface_type") { tmp.assign(d.surface_type, d.surface_type + d.num_surfaces); v = &tmp; }
  else if (nm == "surface_dir") { tmp.assign(d.surface_dir, d.surface_dir + d.num_surfaces); v = &tmp; }
  else if (k->prepared && nm == "nearest_surf") v = &k->s.nearest_surf;
  else if (k->prepared && nm == "eeff_direction") v = &k->s.eeff_dir;
  else if (k->prepared && nm == "electron_num") v = &k->s.electron_num;
  else if (k->prepared && nm == "hole_num") v = &k->s.hole_num;
  else if (k->prepared && nm == "refresh_electrons") v = &k->s.desired_e;
  else if (k->prepared && nm == "refresh_holes") v = &k->s.desired_h;
  else return MCB200_ERR_ARG;
  return copy_out(*v, out, n, needed);
}

int mcb200_deck_double_array(const mcb200_deck *k, const char *name, double *out, size_t n, size_t *needed) {
  if (!k || !name) return MCB200_ERR_ARG;
  if (!k->loaded) return MCB200_ERR_STATE;
  const Deck &d = k->d;
  const DeckScaled &s = k->s;
  const std::string nm(name);
  const std::vector<double> *v = nullptr;
  std::vector<double> tmp;
  if (nm == "lx_m") v = &d.lx_m;
  else if (nm == "ly_m") v = &d.ly_m;
  else if (nm == "lz_m") v = &d.lz_m;
  else if (nm == "donor_m3") v = &d.donor_m3;
  else if (nm == "acceptor_m3") v = &d.acceptor_m3;
  else if (nm == "contact_vapp_v") { for (const auto &c : d.contacts) tmp.push_back(c.vapp_v); v = &tmp; }
  else if (nm == "contact_phims_v") { for (const auto &c : d.contacts) tmp.push_back(c.phims_v); v = &tmp; }
  else if (nm == "surface_pos_nm") { tmp.assign(d.surface_pos_nm, d.surface_pos_nm + d.num_surfaces); v = &tmp; }
  else if (!k->prepared) return MCB200_ERR_ARG;
  else if (nm == "lx") v = &s.lx;
  else if (nm == "ly") v = &s.ly;
  else if (nm == "lz") v = &s.lz;
  else if (nm == "dx") v = &s.dx;
  else if (nm == "dy") v = &s.dy;
  else if (nm == "dz") v = &s.dz;
  else if (nm == "donor") v = &s.donor;
  else if (nm == "acceptor") v = &s.acceptor;
  else if (nm == "volume") v = &s.volume;
  else if (nm == "da") v = &s.da;
  else if (nm == "init_electron_charge") v = &s.init_e_charge;
  else if (nm == "init_hole_charge") v = &s.init_h_charge;
  else if (nm == "contact_vapp") v = &s.vapp;
  else if (nm == "contact_phims") v = &s.phims;
  else if (nm == "surface_pos") { tmp.assign(s.surface_pos, s.surface_pos + d.num_surfaces); v = &tmp; }
  else return MCB200_ERR_ARG;
  return copy_out(*v, out, n, needed);
}

int mcb200_deck_prepare(mcb200_deck *k, const mcb200_ctx *ctx) {
  if (!k || !ctx) return MCB200_ERR_ARG;
  if (!k->loaded) return MCB200_ERR_STATE;
  double u[14];
  if (mcb200_units(ctx, u, 14) != MCB200_OK) return deck_fail(k, MCB200_ERR_STATE, "context has no units");
  if (std::fabs(u[0] - k->d.temperature) > 1e-9)
    return deck_fail(k, MCB200_ERR_ARG, "the context's tables were built at another temperature than the deck's");
  double ni = 0;
  size_t need = 0;
  if (mcb200_copy_table(ctx, "ni", &ni, sizeof(ni), &need) != MCB200_OK)
    return deck_fail(k, MCB200_ERR_STATE, "context has no band tables");
  Units un{};
  un.T0 = u[0]; un.eV0 = u[1]; un.spr0 = u[2]; un.time0 = u[3]; un.conc0 = u[4]; un.field0 = u[5];
  un.scrt0 = u[6]; un.pot0 = u[7];
  try {
    k->s = DeckScaled::build(k->d, un, ni);
    k->prepared = true;
    return MCB200_OK;
  } catch (const std::exception &e) {
    return deck_fail(k, MCB200_ERR_ARG, e.what());
  }
}

int mcb200_apply_deck(mcb200_ctx *ctx, mcb200_deck *k) {
  if (!ctx || !k) return MCB200_ERR_ARG;
  if (!k->prepared) {
    if (int rc = mcb200_deck_prepare(k, ctx)) return rc;
  }
  const Deck &d = k->d;
  const DeckScaled &s = k->s;
  int rc = mcb200_set_mesh(ctx, d.nx, d.ny, d.nz, s.lx.data(), s.ly.data(), s.lz.data(), s.dx.data(), s.dy.data(),
                           s.dz.data());
  if (rc) return deck_fail(k, rc, std::string("mcb200_set_mesh: ") + mcb200_last_error(ctx));
  const int flags = (d.flag_surface_scatter ? MCB200_FLAG_SURFACE_SCATTER : 0) |
                    (d.flag_surface_impurity ? MCB200_FLAG_SURFACE_IMPURITY : 0) |
                    (d.flag_quantum_correction ? MCB200_FLAG_QUANTUM : 0);
  rc = mcb200_set_cells(ctx, d.motion.data(), d.attached_contact.data(), d.in_surf.data(), s.nearest_surf.data(),
                        d.surface_dir, d.num_surfaces, s.da.data(), flags);
  if (rc) return deck_fail(k, rc, std::string("mcb200_set_cells: ") + mcb200_last_error(ctx));
  if (d.flag_quantum_correction) {  // set up now, on from quantum_start_step (mcb200_run_deck)
    mcb200_quantum_params q{};
    for (int a = 0; a < 3; ++a) {
      q.ratio[a] = d.qc_ratio[a];
      q.theta[a] = s.qc_theta[a];
    }
    q.eb = s.qc_eb;
    rc = mcb200_set_quantum_correction(ctx, &q, d.material.data(), d.quantum_region.data(), 0);
    if (rc) return deck_fail(k, rc, std::string("mcb200_set_quantum_correction: ") + mcb200_last_error(ctx));
  }
  const std::vector<int32_t> planes = contact_planes(d);
  rc = mcb200_set_device(ctx, d.material.data(), s.donor.data(), s.acceptor.data(), (int)d.contacts.size(),
                         s.vapp.data(), s.phims.data(), (int)(planes.size() / 7), planes.data());
  if (rc) return deck_fail(k, rc, std::string("mcb200_set_device: ") + mcb200_last_error(ctx));
  return MCB200_OK;
}

int mcb200_seed_deck(mcb200_ctx *ctx, mcb200_deck *k, uint64_t seed) {
  if (!ctx || !k) return MCB200_ERR_ARG;
  if (!k->prepared) return deck_fail(k, MCB200_ERR_STATE, "mcb200_seed_deck before mcb200_apply_deck");
  const Deck &d = k->d;
  const DeckScaled &s = k->s;
  // init_particle_data (src/particle_init.cpp:112-219): per carrier type,
  // cells in (i, k, j) order, each silicon cell's carriers sharing its
  // neutral charge equally
  for (int type = 0; type < 2; ++type) {
    std::vector<int32_t> cell_of;
    std::vector<double> charge;
    for (int i = 0; i < d.nx; ++i)
      for (int kk = 0; kk < d.nz; ++kk)
        for (int j = 0; j < d.ny; ++j) {
          const int c = d.cell(i, j, kk);
          if (d.material[c] != kMatSilicon) continue;
          const int pnum = type == 0 ? s.electron_num[c] : s.hole_num[c];
          // restarted cells away from the contacts keep the file's charge
          // (electrons negative), src/particle_init.cpp:157-178
          const bool restarted = d.flag_restart && d.attached_contact[c] <= 0;
          if (restarted && pnum == 0) continue;
          const double q = restarted ? (type == 0 ? -s.restart_e_charge[c] : s.restart_h_charge[c]) / pnum
                                     : (type == 0 ? s.init_e_charge[c] : s.init_h_charge[c]) / pnum;
          for (int p = 0; p < pnum; ++p) {
            cell_of.push_back(c);
            charge.push_back(q);
          }
        }
    const int rc = mcb200_seed_particles(ctx, cell_of.size(), cell_of.data(), charge.data(), type, seed);
    if (rc) return deck_fail(k, rc, std::string("mcb200_seed_particles: ") + mcb200_last_error(ctx));
  }
  return MCB200_OK;
}

}  // extern "C"
