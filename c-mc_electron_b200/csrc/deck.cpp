// deck.cpp -- input.txt / lgrid.txt / ldg.txt readers and the cell data
// derived from them (see deck.h for the reference routines each step
// restates).
#include "deck.h"

#include <cmath>
#include <cstdlib>
#include <fstream>
#include <map>
#include <sstream>

namespace mcb200 {
namespace {

std::string trim(const std::string &s) {
  const size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
  return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

// input.txt: `key = value` lines, '#' starts a comment (the reading of
// Trilinos_Util::InputFileReader used for the decks in finfet/input.txt).
struct KeyValues {
  std::map<std::string, std::string> kv;
  explicit KeyValues(const std::string &path) {
    std::ifstream in(path);
    if (!in) throw DeckError("cannot open input file " + path);
    std::string line;
    while (std::getline(in, line)) {
      const size_t hash = line.find('#');
      if (hash != std::string::npos) line = line.substr(0, hash);
      const size_t eq = line.find('=');
      if (eq == std::string::npos) continue;
      const std::string k = trim(line.substr(0, eq)), v = trim(line.substr(eq + 1));
      if (!k.empty()) kv[k] = v;
    }
  }
  const std::string *find(const char *k) const {
    auto it = kv.find(k);
    return it == kv.end() ? nullptr : &it->second;
  }
  int get(const char *k, int d) const { const auto *v = find(k); return v ? std::atoi(v->c_str()) : d; }
  double get(const char *k, double d) const { const auto *v = find(k); return v ? std::atof(v->c_str()) : d; }
  bool get(const char *k, bool d) const {
    const auto *v = find(k);
    return v ? (std::atoi(v->c_str()) != 0 || *v == "true") : d;
  }
  std::string get(const char *k, const char *d) const { const auto *v = find(k); return v ? *v : std::string(d); }
};

std::string dir_of(const std::string &path) {
  const size_t s = path.find_last_of('/');
  return s == std::string::npos ? std::string(".") : path.substr(0, s);
}
std::string resolve(const std::string &base, const std::string &name) {
  if (!name.empty() && name[0] == '/') return name;
  return base + "/" + name;
}

// read_grid_file, src/mcmodel.cpp:4595-4693: per axis a count, then the
// node coordinates in micrometres.
void read_grid(const std::string &path, Deck &d) {
  std::ifstream in(path);
  if (!in) throw DeckError("cannot open grid file " + path);
  std::vector<double> *axes[3] = {&d.lx_m, &d.ly_m, &d.lz_m};
  for (auto *ax : axes) {
    int n = 0;
    if (!(in >> n) || n < 2) throw DeckError("bad node count in " + path);
    ax->resize(n);
    for (int i = 0; i < n; ++i) {
      double pos;
      if (!(in >> pos)) throw DeckError("short grid file " + path);
      (*ax)[i] = pos * 1e-6;
    }
  }
  d.nx = (int)d.lx_m.size() - 1;
  d.ny = (int)d.ly_m.size() - 1;
  d.nz = (int)d.lz_m.size() - 1;
  if (d.nx > 1023 || d.ny > 1023 || d.nz > 1023) throw DeckError("more than 1023 cells along an axis");
}

// distance2index, src/mcmodel.cpp:4168-4176: the node at `pos` nanometres.
int node_index(double pos, const std::vector<double> &cut) {
  for (size_t i = 0; i < cut.size(); ++i)
    if (std::fabs(pos - cut[i] * 1e9) < 1e-4) return (int)i;
  std::ostringstream os;
  os << "coordinate " << pos << " nm is not on a grid line";
  throw DeckError(os.str());
}

struct Cmd {
  int type = 0;
  int range[6] = {0, 0, 0, 0, 0, 0};
  double dbl = 0;
  int ip[6] = {0, 0, 0, 0, 0, 0};
};

// The device script, read_device_file (src/mcmodel.cpp:4190-4479).
class DeviceScript {
 public:
  DeviceScript(const std::string &path, Deck &d) : d_(d), in_(path) {
    if (!in_) throw DeckError("cannot open device file " + path);
  }
  std::vector<Cmd> read() {
    static const std::map<std::string, int> op = {
        {"donor", 1}, {"acceptor", 2}, {"region", 3}, {"motioncube", 4}, {"attachcontact", 5}, {"contact", 6},
        {"motionplane", 7}, {"parnumber", 8}, {"default_par_number", 9}, {"ScatterArea", 12}, {"VsVdVg", 13},
        {"vgrange", 14}, {"ep_parm", 15}, {"surfaces", 16}, {"surface_scatter_range", 17}, {"quantumRegion", 18}};
    static const std::map<std::string, int> dir = {{"UP", 0}, {"DOWN", 1}, {"LEFT", 2},
                                                   {"RIGHT", 3}, {"FRONT", 4}, {"BACK", 5}};
    static const std::map<std::string, int> motion = {{"PASS", 1},     {"REFLECT", 2}, {"SCATTOX", 3},
                                                      {"PERIOD", 4},   {"GENERATE", 5}, {"CATCH", 6},
                                                      {"CATCHGATE", 7}, {"GENREF", 8}};
    static const std::map<std::string, int> regions = {{"VACUUM", kMatVacuum}, {"OXIDE", kMatOxide},
                                                       {"SILICON", kMatSilicon}, {"IGZO", kMatIgzo}};
    auto lookup = [](const std::map<std::string, int> &m, const std::string &k) {
      auto it = m.find(k);
      return it == m.end() ? 0 : it->second;  // std::map::operator[] default
    };
    std::vector<Cmd> cmds;
    std::string word;
    for (;;) {
      if (!(in_ >> word)) throw DeckError("device file ends without `end`");
      if (word == "end") break;
      Cmd c;
      c.type = lookup(op, word);
      switch (c.type) {
        case 1:
        case 2:
          cube(c.range);
          c.dbl = number<double>();
          break;
        case 3: {
          cube(c.range);
          c.ip[0] = lookup(regions, token());
          if (c.ip[0] == kMatSilicon) { c.ip[1] = d_.default_e; c.ip[2] = d_.default_h; }
          else if (c.ip[0] == kMatIgzo) { c.ip[1] = d_.default_e; c.ip[2] = d_.default_e; }
          break;
        }
        case 7:
          cube(c.range);
          c.ip[0] = lookup(dir, token());
          c.ip[1] = lookup(motion, token());
          break;
        case 4:
          cube(c.range);
          for (int i = 0; i < 6; ++i) c.ip[i] = lookup(motion, token());
          break;
        case 5:
        case 12:
          cube(c.range);
          c.ip[0] = number<int>();
          break;
        case 8:
          cube(c.range);
          c.ip[0] = number<int>();
          c.ip[1] = number<int>();
          break;
        case 9:
          d_.default_e = number<int>();
          d_.default_h = number<int>();
          break;
        case 6: {
          DeckContact ct;
          ct.nplanes = number<int>();
          ct.phims_v = number<double>();
          if (ct.nplanes < 0 || ct.nplanes > kMaxContactPlanes) throw DeckError("contact with too many planes");
          for (int p = 0; p < ct.nplanes; ++p) cube(ct.plane[p]);
          ct.vapp_v = number<double>();
          if ((int)d_.contacts.size() >= 16) throw DeckError("more than 16 contacts");
          d_.contacts.push_back(ct);
          break;
        }
        case 13:
          for (int i = 0; i < 4; ++i) number<double>();  // Vs Vd Vg phi_top: unused by the transport
          break;
        case 14: {
          const double a = number<double>(), b = number<double>(), e = number<double>(), f = number<double>();
          node_index(a, d_.ly_m); node_index(b, d_.ly_m);  // gate / oxide positions must lie on grid lines
          node_index(e, d_.lx_m); node_index(f, d_.lx_m);
          break;
        }
        case 15:  // ep_parm: quantum-correction window (src/mcmodel.cpp:4549-4556)
          for (int a = 0; a < 3; ++a) {
            d_.qc_ratio[a] = number<double>();
            d_.qc_theta_nm[a] = number<double>();
          }
          d_.qc_eb_v = number<double>();
          break;
        case 16:
          d_.num_surfaces = number<int>();
          if (d_.num_surfaces < 0 || d_.num_surfaces > 30) throw DeckError("more than 30 surfaces");
          for (int i = 0; i < d_.num_surfaces; ++i) {
            d_.surface_type[i] = number<int>();
            d_.surface_pos_nm[i] = number<double>();
            d_.surface_dir[i] = number<int>();
          }
          break;
        case 17:
        case 18:
          cube(c.range);
          break;
        default:
          break;  // an unknown word: the reference reads the next word as a command
      }
      cmds.push_back(c);
    }
    return cmds;
  }

 private:
  std::string token() {
    std::string s;
    if (!(in_ >> s)) throw DeckError("device file ends inside a command");
    return s;
  }
  template <typename T>
  T number() {
    T v{};
    if (!(in_ >> v)) throw DeckError("device file: a number was expected");
    return v;
  }
  // get_cube_range, src/mcmodel.cpp:4178-4188
  void cube(int *idx) {
    double p[6];
    for (double &v : p) v = number<double>();
    idx[0] = node_index(p[0], d_.lx_m);
    idx[1] = node_index(p[1], d_.lx_m);
    idx[2] = node_index(p[2], d_.ly_m);
    idx[3] = node_index(p[3], d_.ly_m);
    idx[4] = node_index(p[4], d_.lz_m);
    idx[5] = node_index(p[5], d_.lz_m);
  }
  Deck &d_;
  std::ifstream in_;
};

// init_vector_entry, src/set_user_defined_data.cpp:3-51: cells [i0,i1) x
// [j0,j1) x [k0,k1) of a non-empty box inside the mesh.
template <typename T>
void fill_box(const Deck &d, const int *r, T v, std::vector<T> &a) {
  if (!(r[0] >= 0 && r[1] <= d.nx && r[0] < r[1] && r[4] >= 0 && r[5] <= d.nz && r[4] < r[5] && r[2] >= 0 &&
        r[3] <= d.ny && r[2] < r[3]))
    return;  // the reference prints "Overflow or ijk error" and skips
  for (int i = r[0]; i < r[1]; ++i)
    for (int k = r[4]; k < r[5]; ++k)
      for (int j = r[2]; j < r[3]; ++j) a[d.cell(i, j, k)] = v;
}

// SetMRCube, src/set_user_defined_data.cpp:54-85.
void motion_cube(Deck &d, const int *r, const int *mr) {
  if (!(r[0] >= 0 && r[1] <= d.nx && r[0] < r[1] && r[4] >= 0 && r[5] <= d.nz && r[4] < r[5] && r[2] >= 0 &&
        r[3] <= d.ny && r[2] < r[3]))
    return;
  for (int i = r[0]; i < r[1]; ++i)
    for (int k = r[4]; k < r[5]; ++k)
      for (int j = r[2]; j < r[3]; ++j)
        for (int f = 0; f < 6; ++f) d.motion[(size_t)d.cell(i, j, k) * 6 + f] = mr[f];
}

// SetMRPlane, src/set_user_defined_data.cpp:87-183: the rule for particles
// hitting the plane in direction idn, stored on the cell face the plane is.
void motion_plane(Deck &d, const int *r, int idn, int mr) {
  const int bi = r[0], ei = r[1], bj = r[2], ej = r[3], bk = r[4], ek = r[5];
  if (!(bi >= 0 && ei <= d.nx && bi <= ei && bk >= 0 && ek <= d.nz && bk <= ek && bj >= 0 && ej <= d.ny &&
        bj <= ej))
    return;
  auto set = [&](int i, int j, int k, int f) { d.motion[(size_t)d.cell(i, j, k) * 6 + f] = mr; };
  if (bi == ei) {
    if (bj == ej || bk == ek) return;  // "Must be a Plane"
    if (idn == 0) {                    // UP
      if (bi <= d.nx - 1)
        for (int k = bk; k < ek; ++k)
          for (int j = bj; j < ej; ++j) set(bi, j, k, 0);
    } else if (idn == 1) {  // DOWN
      if (bi > 0)
        for (int k = bk; k < ek; ++k)
          for (int j = bj; j < ej; ++j) set(bi - 1, j, k, 1);
    }
  } else if (bj == ej) {
    if (bk == ek) return;
    if (idn == 2) {  // LEFT
      if (bj >= 0 && bj <= d.ny - 1)
        for (int k = bk; k < ek; ++k)
          for (int i = bi; i < ei; ++i) set(i, bj, k, 2);
    } else if (idn == 3) {  // RIGHT
      if (bj - 1 >= 0 && bj - 1 <= d.ny - 1)
        for (int k = bk; k < ek; ++k)
          for (int i = bi; i < ei; ++i) set(i, bj - 1, k, 3);
    }
  } else if (bk == ek) {
    if (idn == 5) {  // BACK
      if (bk > 0)
        for (int i = bi; i < ei; ++i)
          for (int j = bj; j < ej; ++j) set(i, j, bk - 1, 5);
    } else if (idn == 4) {  // FRONT (the reference requires bk < nz - 1)
      if (bk < d.nz - 1)
        for (int i = bi; i < ei; ++i)
          for (int j = bj; j < ej; ++j) set(i, j, bk, 4);
    }
  }
}

}  // namespace

Deck Deck::load(const std::string &input_path) {
  Deck d;
  d.input_path = input_path;
  d.base_dir = dir_of(input_path);
  const KeyValues kv(input_path);
  d.temperature = kv.get("Temperature", 300.0);
  d.grid_file = kv.get("gridFile", "lgrid.txt");
  d.device_file = kv.get("device_file_name", "ldg.txt");
  d.total_step = kv.get("total_step", 100000);
  d.electron_number = kv.get("ElectronNumber", 100000);
  d.hole_number = kv.get("HoleNumber", 100000);
  d.flag_nonlinear_poisson = kv.get("NonLinearPoisson", false);
  d.flag_multiple_refresh = kv.get("Flag_MultipleRefresh", false);
  d.flag_quantum_correction = kv.get("Flag_QuantumCorrection", false);
  d.quantum_start_step = kv.get("quantum_start_step", 20);
  d.flag_surface_scatter = kv.get("Flag_SurfaceScatter", true);
  d.flag_surface_roughness = kv.get("Flag_SurfaceRoughnessScatter", true);
  d.flag_surface_phonon = kv.get("Flag_SurfacePhononScatter", true);
  d.flag_surface_impurity = kv.get("Flag_SurfaceImpurityScatter", false);
  d.flag_compute_potential = kv.get("Flag_compute_potential", true);
  d.flag_compute_heat = kv.get("Flag_compute_heat", false);
  d.heat_steps = kv.get("heat_steps", 20000);
  d.dt_s = kv.get("dt", 1e-16);
  d.flag_restart = kv.get("Flag_restart", false);
  d.restart_step = kv.get("restart_step", 0);
  d.restart_file = kv.get("restart_filename", "nosuchname");
  d.stat_step = kv.get("stat_step", 5000);
  d.stat_heat_step = kv.get("stat_heat_step", 5000);
  d.output_dir = kv.get("OutPut_DIR", "../data");
  d.mr_step = kv.get("mr_step", 10);
  if (d.stat_step <= 0 || d.mr_step <= 0 || d.dt_s <= 0) throw DeckError("stat_step, mr_step and dt must be positive");

  read_grid(resolve(d.base_dir, d.grid_file), d);
  const int cells = d.cells();
  d.material.assign(cells, 0);
  d.desired_e.assign(cells, 0);
  d.desired_h.assign(cells, 0);
  d.attached_contact.assign(cells, 0);
  d.scatter_type.assign(cells, 0);
  d.in_surf.assign(cells, 0);
  d.quantum_region.assign(cells, 0);
  d.motion.assign((size_t)cells * 6, 0);
  d.donor_m3.assign(cells, 0.0);
  d.acceptor_m3.assign(cells, 0.0);

  DeviceScript script(resolve(d.base_dir, d.device_file), d);
  const std::vector<Cmd> cmds = script.read();
  // init_by_user_input, src/mcmodel.cpp:3065-3153
  for (const Cmd &c : cmds) {
    switch (c.type) {
      case 1: fill_box(d, c.range, c.dbl, d.donor_m3); break;
      case 2: fill_box(d, c.range, c.dbl, d.acceptor_m3); break;
      case 3:
        fill_box(d, c.range, c.ip[0], d.material);
        fill_box(d, c.range, c.ip[1], d.desired_e);
        fill_box(d, c.range, c.ip[2], d.desired_h);
        break;
      case 4: motion_cube(d, c.range, c.ip); break;
      case 5: fill_box(d, c.range, c.ip[0], d.attached_contact); break;
      case 7: motion_plane(d, c.range, c.ip[0], c.ip[1]); break;
      case 8:
        fill_box(d, c.range, c.ip[0], d.desired_e);
        fill_box(d, c.range, c.ip[1], d.desired_h);
        break;
      case 12: fill_box(d, c.range, c.ip[0], d.scatter_type); break;
      case 17:  // surface_scatter_range; the reference falls through to quantumRegion
        fill_box(d, c.range, 1, d.in_surf);
        fill_box(d, c.range, 1, d.quantum_region);
        break;
      case 18: fill_box(d, c.range, 1, d.quantum_region); break;
      default: break;
    }
  }
  return d;
}

DeckScaled DeckScaled::build(const Deck &d, const Units &u, double ni) {
  DeckScaled s;
  const double spr0 = u.spr0;
  // scaling(): node coordinates and the widths read in metres, each divided by spr0
  auto scale_axis = [&](const std::vector<double> &m, std::vector<double> &l, std::vector<double> &w) {
    l.resize(m.size());
    w.resize(m.size() - 1);
    for (size_t i = 0; i < m.size(); ++i) l[i] = m[i] / spr0;
    for (size_t i = 1; i < m.size(); ++i) w[i - 1] = (m[i] - m[i - 1]) / spr0;
  };
  scale_axis(d.lx_m, s.lx, s.dx);
  scale_axis(d.ly_m, s.ly, s.dy);
  scale_axis(d.lz_m, s.lz, s.dz);
  s.dt = d.dt_s / u.time0;
  for (const DeckContact &c : d.contacts) {
    s.vapp.push_back(c.vapp_v / u.pot0);
    s.phims.push_back(c.phims_v / u.pot0);
  }
  for (int i = 0; i < d.num_surfaces; ++i) s.surface_pos[i] = d.surface_pos_nm[i] * 1e-9 / spr0;
  for (int a = 0; a < 3; ++a) s.qc_theta[a] = d.qc_theta_nm[a] / (1e9 * spr0);
  s.qc_eb = d.qc_eb_v / u.pot0;
  const int cells = d.cells();
  s.donor.resize(cells);
  s.acceptor.resize(cells);
  s.volume.resize(cells);
  s.da.resize(cells);
  s.init_e_charge.assign(cells, 0.0);
  s.init_h_charge.assign(cells, 0.0);
  for (int c = 0; c < cells; ++c) {
    s.donor[c] = d.donor_m3[c] / u.conc0;
    s.acceptor[c] = d.acceptor_m3[c] / u.conc0;
  }
  // init_cell_data: volumes, |doping|, and the neutral carrier charge of each
  // silicon cell, summed in the reference's loop order (i, k, j)
  for (int i = 0; i < d.nx; ++i)
    for (int k = 0; k < d.nz; ++k)
      for (int j = 0; j < d.ny; ++j) {
        const int c = d.cell(i, j, k);
        s.volume[c] = s.dx[i] * s.dy[j] * s.dz[k];
        s.da[c] = s.donor[c] + s.acceptor[c];
      }
  for (int i = 0; i < d.nx; ++i)
    for (int k = 0; k < d.nz; ++k)
      for (int j = 0; j < d.ny; ++j) {
        const int c = d.cell(i, j, k);
        if (d.material[c] != kMatSilicon) continue;
        const double dope = s.donor[c] - s.acceptor[c], vol = s.volume[c];
        if (dope > 0) {
          s.init_e_charge[c] = -dope * vol;
          s.init_h_charge[c] = (ni * ni / dope) * vol;
        } else if (dope < 0) {
          s.init_e_charge[c] = (ni * ni / dope) * vol;
          s.init_h_charge[c] = -dope * vol;
        } else {
          s.init_e_charge[c] = -ni * vol;
          s.init_h_charge[c] = ni * vol;
        }
        s.sum_e += s.init_e_charge[c];
        s.sum_h += s.init_h_charge[c];
      }
  // init_surface_roughness: nearest Si/oxide surface of each cell (from the
  // cell's low node) and the field component normal to it
  s.nearest_surf.assign(cells, 0);
  s.eeff_dir.assign(cells, 0);
  if (d.flag_surface_scatter) {
    for (int i = 0; i < d.nx; ++i)
      for (int k = 0; k < d.nz; ++k)
        for (int j = 0; j < d.ny; ++j) {
          const int c = d.cell(i, j, k);
          double dist = 1e99;
          int nearest = 0;
          for (int q = 0; q < d.num_surfaces; ++q) {
            const double pos = s.surface_pos[q];
            if (d.surface_type[q] == 0 && dist > std::fabs(s.lx[i] - pos)) { dist = std::fabs(s.lx[i] - pos); nearest = q; }
            if (d.surface_type[q] == 1 && dist > std::fabs(s.ly[j] - pos)) { dist = std::fabs(s.ly[j] - pos); nearest = q; }
            if (d.surface_type[q] == 2 && dist > std::fabs(s.lz[k] - pos)) { dist = std::fabs(s.lz[k] - pos); nearest = q; }
          }
          s.nearest_surf[c] = nearest;
          s.eeff_dir[c] = d.surface_type[nearest];
        }
  }
  // compute_par_num: carriers per silicon cell from its share of the total
  // charge, and the refresh targets raised to at least that (and the default)
  s.electron_num.assign(cells, 0);
  s.hole_num.assign(cells, 0);
  s.desired_e = d.desired_e;
  s.desired_h = d.desired_h;
  for (int c = 0; c < cells; ++c) {
    if (d.material[c] != kMatSilicon) continue;
    s.electron_num[c] = int(1e-10 + s.init_e_charge[c] / s.sum_e * d.electron_number) + 1;
    s.hole_num[c] = int(1e-10 + s.init_h_charge[c] / s.sum_h * d.hole_number) + 1;
    if (s.electron_num[c] > s.desired_e[c]) s.desired_e[c] = s.electron_num[c];
    if (s.hole_num[c] > s.desired_h[c]) s.desired_h[c] = s.hole_num[c];
    if (s.desired_e[c] < d.default_e) s.desired_e[c] = d.default_e;
    if (s.desired_h[c] < d.default_h) s.desired_h[c] = d.default_h;
  }
  // Flag_restart (init_particle_data, src/particle_init.cpp:130-134, with
  // read_par_info_for_restart, src/mcmodel.cpp:853-889): the restart file's
  // lines "i j k |q|_e n_e |q|_h n_h", ended by a negative i, replace the
  // carrier counts of the cells they name (the refresh targets keep theirs)
  // and give the charges a restarted silicon cell away from the contacts
  // shares among its carriers.  Cells off the mesh are skipped.
  if (d.flag_restart) {
    const std::string path = resolve(d.base_dir, d.restart_file);
    std::ifstream f(path);
    if (!f) throw DeckError("cannot open the restart file " + path);
    s.restart_e_charge.assign(cells, 0.0);
    s.restart_h_charge.assign(cells, 0.0);
    for (;;) {
      int i = 0, j = 0, k = 0;
      if (!(f >> i >> j >> k)) throw DeckError("restart file " + path + " ends before its -1 line");
      if (i < 0) break;
      double c1 = 0, c2 = 0;
      int n1 = 0, n2 = 0;
      if (!(f >> c1 >> n1 >> c2 >> n2)) throw DeckError("restart file " + path + ": short line");
      if (i >= d.nx || j < 0 || j >= d.ny || k < 0 || k >= d.nz) continue;
      const int c = d.cell(i, j, k);
      s.restart_e_charge[c] = c1;
      s.restart_h_charge[c] = c2;
      s.electron_num[c] = n1;
      s.hole_num[c] = n2;
    }
  }
  return s;
}

}  // namespace mcb200
