// driver.cpp -- the self-consistent simulation behind `main input.txt`:
// MeshQuantities::run / density (src/mcmodel.cpp:499-566, :424-467) and
// compute_heat / heat_density (src/heat.cpp:48-160) over the engine's C ABI,
// with the reference's data/ outputs (output_stat, current_scatter_info,
// output_for_restart; src/mcmodel.cpp:756-1161).
//
// Per transport step, as density() orders it: statistics of the store
// (statistic), charge deposition (particle_to_density + compute_cell_charge),
// the Poisson solve and cell fields (compute_field; every poisson_every
// steps, 1 = every step as the reference), surface rates when surface
// scattering is on (GetSurfRoughnessPhononScRate), then the carrier step
// (update_particle).  MultipleRefresh every mr_step steps; outputs every
// stat_step steps, appended to the per-step files as the reference opens
// them (section_current and the first `current` are truncated).
#include <sys/stat.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "mcb200.h"

namespace {

struct RunError : std::runtime_error {
  int code;
  RunError(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

void ok(int rc, mcb200_ctx *c, const char *what) {
  if (rc != MCB200_OK) throw RunError(rc, std::string(what) + ": " + (c ? mcb200_last_error(c) : ""));
}
void deck_ok(int rc, mcb200_deck *d, const char *what) {
  if (rc != MCB200_OK) throw RunError(rc, std::string(what) + ": " + (d ? mcb200_deck_error(d) : ""));
}

std::vector<int32_t> deck_ints(mcb200_deck *d, const char *name) {
  size_t n = 0;
  deck_ok(mcb200_deck_int_array(d, name, nullptr, 0, &n), d, name);
  std::vector<int32_t> v(n);
  deck_ok(mcb200_deck_int_array(d, name, v.data(), n, &n), d, name);
  return v;
}
std::vector<double> deck_doubles(mcb200_deck *d, const char *name) {
  size_t n = 0;
  deck_ok(mcb200_deck_double_array(d, name, nullptr, 0, &n), d, name);
  std::vector<double> v(n);
  deck_ok(mcb200_deck_double_array(d, name, v.data(), n, &n), d, name);
  return v;
}

// input.txt keys the reference does not read: run-time choices of this engine.
struct Extras {
  double delta_nm = 0.1126755, lambda_nm = 2.0;  // surface roughness (the reference's hard-coded values)
  int poisson_every = 1;
};
Extras read_extras(const std::string &path) {
  Extras e;
  std::ifstream in(path);
  std::string line;
  while (std::getline(in, line)) {
    const size_t hash = line.find('#');
    if (hash != std::string::npos) line = line.substr(0, hash);
    const size_t eq = line.find('=');
    if (eq == std::string::npos) continue;
    std::string k = line.substr(0, eq), v = line.substr(eq + 1);
    k.erase(0, k.find_first_not_of(" \t"));
    k.erase(k.find_last_not_of(" \t\r") + 1);
    if (k == "surface_roughness_delta_nm") e.delta_nm = std::atof(v.c_str());
    else if (k == "surface_roughness_lambda_nm") e.lambda_nm = std::atof(v.c_str());
    else if (k == "poisson_step") e.poisson_every = std::max(1, std::atoi(v.c_str()));
  }
  return e;
}

struct Run {
  mcb200_ctx *ctx = nullptr;
  mcb200_deck *deck = nullptr;
  mcb200_deck_info info{};
  mcb200_run_options opt{};
  mcb200_run_report *rep = nullptr;
  std::string data_dir;
  double u[14];
  int nx = 0, ny = 0, nz = 0, cells = 0, nodes = 0;
  std::vector<int32_t> refresh_e, refresh_h, eeff;
  std::vector<double> node_volume, saved_e_charge, saved_h_charge, pot_avg, qc_avg;
  mcb200_surface_params surf{};
  int poisson_every = 1;
  uint64_t seed = 1;
  bool heat = false;
  bool qc_on = false;  // the quantum correction has been switched on

  double T0() const { return u[0]; }
  double spr0() const { return u[2]; }
  double time0() const { return u[3]; }
  double conc0() const { return u[4]; }
  double pot0() const { return u[7]; }
  double curr0() const { return u[12]; }

  std::string file(const char *prefix, int step) const {
    std::ostringstream os;
    os << data_dir << "/" << prefix << step;
    return os.str();
  }

  using clock = std::chrono::steady_clock;
  clock::time_point mark = clock::now();
  // wall time since the last lap into report->phase_s[phase] (after the
  // GPU has finished the phase when profiling phases)
  void lap(int phase) {
    if (opt.profile_phases) ok(mcb200_sync(ctx), ctx, "mcb200_sync");
    const clock::time_point now = clock::now();
    rep->phase_s[phase] += std::chrono::duration<double>(now - mark).count();
    mark = now;
  }

  // One step of density() (heat == false) or heat_density() (heat == true).
  void density(int step) {
    mark = clock::now();
    ok(mcb200_stat_accumulate(ctx), ctx, "mcb200_stat_accumulate");
    lap(0);
    ok(mcb200_deposit(ctx), ctx, "mcb200_deposit");
    lap(1);
    // compute_field applies the quantum correction from quantum_start_step on (src/mcmodel.cpp:2249)
    if (!heat && info.flag_quantum_correction && !qc_on && step >= info.quantum_start_step) {
      ok(mcb200_set_quantum_correction(ctx, nullptr, nullptr, nullptr, 1), ctx, "mcb200_set_quantum_correction");
      qc_on = true;
    }
    if (!heat && info.flag_compute_potential && step % poisson_every == 0)  // statistics stay on the device
      ok(mcb200_solve_poisson(ctx, opt.poisson_rel_tol > 0 ? opt.poisson_rel_tol : 1e-10, 20000, nullptr, nullptr),
         ctx, "mcb200_solve_poisson");
    lap(2);
    if (info.flag_surface_scatter) ok(mcb200_surface_rates(ctx, &surf, eeff.data()), ctx, "mcb200_surface_rates");
    lap(3);
    ok(mcb200_step(ctx, (uint32_t)(heat ? 0x80000000u + step : step), seed, info.dt), ctx, "mcb200_step");
    lap(4);
  }

  void refresh(int step) {
    if (!info.flag_multiple_refresh || step % info.mr_step != info.mr_step - 1) return;
    mark = clock::now();
    // (the count of new particles is not asked for: reading it would make
    // the host wait for the GPU)
    ok(mcb200_multiple_refresh(ctx, refresh_e.data(), refresh_h.data(), (uint32_t)(heat ? 0x80000000u + step : step),
                               seed, nullptr),
       ctx, "mcb200_multiple_refresh");
    rep->refreshes += 1;
    lap(5);
  }

  // output_stat + current_scatter_info + output_for_restart for the window
  // that ends at `step` (stat_step steps), then a new window.
  void output(int step, int window) {
    mark = clock::now();
    if (opt.write_outputs) write_outputs(step, window);
    ok(mcb200_reset_tallies(ctx), ctx, "mcb200_reset_tallies");
    ok(mcb200_stat_begin(ctx, window), ctx, "mcb200_stat_begin");
    lap(6);
  }

  void write_outputs(int step, int window) {
    const double dt = info.dt, pot0v = pot0(), curr0v = curr0(), velo0 = spr0() / time0(), conc0v = conc0();
    std::vector<uint64_t> counters(MCB200_NUM_COUNTERS);
    std::vector<double> contact(16 * 6), lcur(ny + 1), rcur(ny + 1), he(nodes), hh(nodes);
    ok(mcb200_get_tallies(ctx, counters.data(), contact.data(), lcur.data(), rcur.data(), he.data(), hh.data()), ctx,
       "mcb200_get_tallies");
    {  // current (appended per window) and section_current<step>
      std::ofstream f(data_dir + "/current", std::ios::app);
      f << "step = " << step << "\n";
      for (int c = 0; c < info.n_contacts; ++c) {
        const double *t = &contact[6 * c];
        f << "icont = " << c << "\n"
          << "CharGen = " << t[1] << ' ' << "NumParGen = " << (long long)t[0] << ' ' << "CharCatch = " << t[4] << ' '
          << "NumParCatch = " << (long long)t[3] << "\n"
          << "EnergyGen= " << t[2] << "\n"
          << "EnergyCatch= " << t[5] << "\n"
          << "EnergyCurrent= " << (t[5] - t[2]) / (dt * window) * pot0v << "\n"
          << "Current = " << (t[1] - t[4]) / (dt * window) * curr0v * 1e-2 << "\n";
      }
      f << "times of phonon scatter : " << counters[MCB200_CNT_PHONON] << "\n"
        << "times of impurity scatter : " << counters[MCB200_CNT_IMPURITY] << "\n";
      std::ofstream s(file("section_current", step));
      for (int j = 0; j <= ny; ++j)
        s << j << ' ' << rcur[j] / (dt * window) * curr0v << ' ' << lcur[j] / (dt * window) * curr0v << ' '
          << (rcur[j] - lcur[j]) / (dt * window) * curr0v << "\n";
    }
    auto stat = [&](const char *name, size_t n) {
      std::vector<double> v(n);
      ok(mcb200_stat_get(ctx, name, v.data(), n), ctx, name);
      return v;
    };
    const std::vector<double> count = stat("cell_count", cells), pot = stat("pot_sum", nodes),
                              qc_pot = stat("qc_pot_sum", nodes);
    auto cidx = [&](int i, int j, int k) { return ((size_t)j * nx + i) * nz + k; };
    auto nidx = [&](int i, int j, int k) { return ((size_t)j * (nx + 1) + i) * (nz + 1) + k; };
    {
      std::ofstream f(file("electron_num", step), std::ios::app);
      for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
          for (int k = 0; k < nz; ++k) f << i << ' ' << j << ' ' << k << ' ' << count[cidx(i, j, k)] / window << "\n";
    }
    pot_avg.assign(nodes, 0.0);
    qc_avg.assign(nodes, 0.0);
    {
      std::ofstream f(file("pot", step), std::ios::app), q(file("qc_pot", step), std::ios::app);
      for (int i = 0; i <= nx; ++i)
        for (int k = 0; k <= nz; ++k)
          for (int j = 0; j <= ny; ++j) {
            const size_t p = nidx(i, j, k);
            pot_avg[p] = pot[p] / window;
            qc_avg[p] = qc_pot[p] / window;
            f << i << ' ' << j << ' ' << k << ' ' << pot_avg[p] * pot0v << "\n";
            q << i << ' ' << j << ' ' << k << ' ' << qc_avg[p] * pot0v << "\n";
          }
    }
    const char *names[2] = {"Electron", "Hole"};
    const char *pre[2] = {"electron_", "hole_"};
    std::vector<double> qsum[2];
    for (int t = 0; t < 2; ++t) {
      const std::string p(pre[t]);
      const std::vector<double> qvx = stat((p + "qvx").c_str(), nodes), qvy = stat((p + "qvy").c_str(), nodes),
                                qvz = stat((p + "qvz").c_str(), nodes), qe = stat((p + "qe").c_str(), nodes);
      qsum[t] = stat((p + "q").c_str(), nodes);
      std::vector<double> &saved = t == 0 ? saved_e_charge : saved_h_charge;
      saved.assign(nodes, 0.0);
      std::ofstream f(file(names[t], step), std::ios::app);
      for (int i = 0; i <= nx; ++i)
        for (int k = 0; k <= nz; ++k)
          for (int j = 0; j <= ny; ++j) {
            const size_t n = nidx(i, j, k);
            const double q = qsum[t][n], aq = std::fabs(q);
            double vx = 0, vy = 0, vz = 0, en = 0;
            if (aq > 1e-13) {
              vx = qvx[n] / aq * velo0;
              vy = qvy[n] / aq * velo0;
              vz = qvz[n] / aq * velo0;
              en = qe[n] / aq * pot0v;
            }
            const double dens = node_volume[n] > 1e-13 ? q / node_volume[n] / window * conc0v : 0.0;
            saved[n] = dens;
            f << i << ' ' << j << ' ' << k << ' ' << vx << ' ' << vy << ' ' << vz << ' ' << en << ' ' << dens << "\n";
          }
    }
    if (heat) {
      std::ofstream f(file("heat", step), std::ios::app);
      for (int i = 0; i <= nx; ++i)
        for (int k = 0; k <= nz; ++k)
          for (int j = 0; j <= ny; ++j) {
            const size_t n = nidx(i, j, k);
            const double v1 = std::fabs(qsum[0][n]) > 1e-13 ? he[n] * pot0v / qsum[0][n] : 0.0;
            const double v2 = std::fabs(qsum[1][n]) > 1e-13 ? hh[n] * pot0v / qsum[1][n] : 0.0;
            f << i << ' ' << j << ' ' << k << ' ' << v1 << ' ' << v1 * saved_e_charge[n] << ' ' << v2 << ' '
              << v2 * saved_h_charge[n] << "\n";
          }
      double total = 0;
      for (int n = 0; n < nodes; ++n) total += he[n] + hh[n];
      rep->heat_total += total;
    }
    {  // par_info_restart<step>: per cell |q| and count of each carrier type
      const size_t n = mcb200_num_particles(ctx);
      std::vector<double> pd[8];
      std::vector<int32_t> pi[6];
      std::vector<uint32_t> uid(n);
      for (auto &v : pd) v.resize(n);
      for (auto &v : pi) v.resize(n);
      mcb200_particles hp{pd[0].data(), pd[1].data(), pd[2].data(), pd[3].data(), pd[4].data(), pd[5].data(),
                          pd[6].data(), pd[7].data(), pi[0].data(), pi[1].data(), pi[2].data(), pi[3].data(),
                          pi[4].data(), pi[5].data(), uid.data()};
      size_t got = 0;
      ok(mcb200_download_particles(ctx, &hp, n, &got), ctx, "mcb200_download_particles");
      std::vector<double> ec(cells, 0.0), hc(cells, 0.0);
      std::vector<int> en(cells, 0), hn(cells, 0);
      // summed in uid order: the store's order within a cell varies from run
      // to run (the cell sort's atomics), the file must not
      std::vector<uint32_t> order(got);
      for (size_t q = 0; q < got; ++q) order[q] = (uint32_t)q;
      std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return uid[a] < uid[b]; });
      for (const uint32_t q : order) {
        const size_t c = cidx(pi[0][q], pi[1][q], pi[2][q]);
        if (pi[5][q] == 0) { ec[c] += std::fabs(pd[6][q]); en[c]++; }
        else { hc[c] += std::fabs(pd[6][q]); hn[c]++; }
      }
      std::ofstream f(file("par_info_restart", step), std::ios::app);
      for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
          for (int k = 0; k < nz; ++k) {
            const size_t c = cidx(i, j, k);
            f << i << ' ' << j << ' ' << k << ' ' << ec[c] << ' ' << en[c] << ' ' << hc[c] << ' ' << hn[c] << "\n";
          }
      f << "-1 -1 -1\n";
    }
    // drain current of the window: contact 1 when there are several, else 0
    const int drain = info.n_contacts > 1 ? 1 : 0;
    if (info.n_contacts > 0)
      rep->last_current[0] = (contact[6 * drain + 1] - contact[6 * drain + 4]) / (dt * window) * curr0v * 1e-2;
    rep->windows += 1;
  }

  void go(const char *input_path, int device) {
    deck_ok(mcb200_deck_load(input_path, &deck), deck, "mcb200_deck_load");
    deck_ok(mcb200_deck_get_info(deck, &info), deck, "mcb200_deck_get_info");
    const Extras ex = read_extras(input_path);
    poisson_every = opt.poisson_every > 0 ? opt.poisson_every : ex.poisson_every;
    seed = opt.seed ? opt.seed : 1;
    // tables and context
    const char *tables = opt.table_dir;
    if (!tables) throw RunError(MCB200_ERR_ARG, "no table directory");
    mcb200_ctx *probe = nullptr;
    if (int rc = mcb200_create(tables, info.temperature, -1, 1, &probe)) {
      const std::string m = probe ? mcb200_last_error(probe) : "";
      mcb200_destroy(probe);
      throw RunError(rc, "tables: " + m);
    }
    deck_ok(mcb200_deck_prepare(deck, probe), deck, "mcb200_deck_prepare");
    mcb200_destroy(probe);
    deck_ok(mcb200_deck_get_info(deck, &info), deck, "mcb200_deck_get_info");
    const std::vector<int32_t> en = deck_ints(deck, "electron_num"), hn = deck_ints(deck, "hole_num");
    refresh_e = deck_ints(deck, "refresh_electrons");
    refresh_h = deck_ints(deck, "refresh_holes");
    eeff = deck_ints(deck, "eeff_direction");
    size_t start = 0, target = 0;
    for (size_t c = 0; c < en.size(); ++c) {
      start += (size_t)en[c] + hn[c];
      target += (size_t)refresh_e[c] + refresh_h[c];
    }
    const size_t capacity = std::max(start, target) + std::max(start, target) / 4 + 65536;
    ok(mcb200_create(tables, info.temperature, device, capacity, &ctx), ctx, "mcb200_create");
    if (opt.flight_precision) ok(mcb200_set_flight_precision(ctx, opt.flight_precision), ctx, "precision");
    ok(mcb200_units(ctx, u, 14), ctx, "mcb200_units");
    deck_ok(mcb200_apply_deck(ctx, deck), deck, "mcb200_apply_deck");
    nx = info.nx; ny = info.ny; nz = info.nz;
    cells = nx * ny * nz;
    nodes = (nx + 1) * (ny + 1) * (nz + 1);
    node_volume.resize(nodes);
    ok(mcb200_get_array(ctx, "node_volume", node_volume.data(), nodes), ctx, "node_volume");
    deck_ok(mcb200_seed_deck(ctx, deck, seed), deck, "mcb200_seed_deck");
    rep->initial_particles = mcb200_num_particles(ctx);
    surf.delta = ex.delta_nm * 1e-9 / spr0();
    surf.ail = ex.lambda_nm * 1e-9 / spr0();
    surf.xiph = 12.0; surf.theta = 2.857703; surf.gama = 1.5; surf.nbmod = 2.0;
    surf.npf = -0.6; surf.pft = 0.7; surf.pfn = 0.3; surf.kpha = 3600e-4;
    surf.roughness = info.flag_surface_roughness;
    surf.phonon = info.flag_surface_phonon;
    data_dir = opt.data_dir ? opt.data_dir : "./data";
    if (opt.write_outputs) {
      ::mkdir(data_dir.c_str(), 0755);
      std::ofstream(data_dir + "/current", std::ios::trunc);
    }
    // the first fields: deposit and solve before the first step
    ok(mcb200_deposit(ctx), ctx, "mcb200_deposit");
    if (info.flag_compute_potential) {
      int it = 0;
      double res = 0;
      ok(mcb200_solve_poisson(ctx, 1e-10, 20000, &it, &res), ctx, "mcb200_solve_poisson");
      ok(mcb200_poisson_stats(ctx, nullptr, nullptr, nullptr, 1), ctx, "mcb200_poisson_stats");  // the run's solves only
    }
    uint64_t ps_start = 0;
    ok(mcb200_particle_steps(ctx, &ps_start), ctx, "mcb200_particle_steps");
    ok(mcb200_set_timing(ctx, 1), ctx, "mcb200_set_timing");
    // run(): from restart_step on with Flag_restart (src/mcmodel.cpp:507-518)
    const int first = info.flag_restart ? std::max(0, info.restart_step) : 0;
    const int remaining = std::max(0, info.total_step - first);
    const int steps = opt.max_steps > 0 ? std::min(opt.max_steps, remaining) : remaining;
    const int warm = std::max(0, std::min(opt.warmup_steps, steps));
    ok(mcb200_stat_begin(ctx, info.stat_step), ctx, "mcb200_stat_begin");
    const auto t0 = std::chrono::steady_clock::now();
    auto timed_t0 = t0;
    uint64_t ps0 = 0;
    heat = false;
    std::vector<double> readback(16 * 6);
    double flushed_ms = 0;  // device time of the timed steps when each follows an L2 eviction
    // Each flushed step is bracketed by a pair of marks (slots 2-7: three
    // pairs in turn); a pair is read only when it is about to be reused, so
    // the host stays up to two steps ahead of the device and no step waits
    // for its own launches to be enqueued.
    bool pair_used[3] = {false, false, false};
    auto settle = [&](int pair) {
      if (!pair_used[pair]) return;
      double ms = 0;
      ok(mcb200_elapsed_ms(ctx, 2 + 2 * pair, 3 + 2 * pair, &ms), ctx, "mcb200_elapsed_ms");
      flushed_ms += ms;
      pair_used[pair] = false;
    };
    for (int step = first; step < first + steps; ++step) {
      if (step == first + warm) {  // the timed region starts: device event + engine timing reset
        ok(mcb200_sync(ctx), ctx, "mcb200_sync");
        // one step in ten bracketed by events: the flight's device time without
        // costing the other steps their overlapped launches
        ok(mcb200_set_timing(ctx, 10), ctx, "mcb200_set_timing");
        ok(mcb200_mark(ctx, 0), ctx, "mcb200_mark");
        timed_t0 = std::chrono::steady_clock::now();
        ok(mcb200_particle_steps(ctx, &ps0), ctx, "mcb200_particle_steps");
      }
      const bool flush = opt.flush_l2_bytes > 0 && step >= first + warm;
      const int pair = step % 3;
      if (flush) {
        settle(pair);
        ok(mcb200_flush_l2(ctx, opt.flush_l2_bytes), ctx, "mcb200_flush_l2");
        ok(mcb200_mark(ctx, 2 + 2 * pair), ctx, "mcb200_mark");
      }
      density(step);
      refresh(step);
      if (flush) {
        ok(mcb200_mark(ctx, 3 + 2 * pair), ctx, "mcb200_mark");
        pair_used[pair] = true;
      }
      if (opt.readback_every_step) {
        // this step's contact tallies to the host without waiting; the
        // previous step's are read while this one runs on the GPU
        ok(mcb200_tallies_enqueue(ctx, step & 1), ctx, "mcb200_tallies_enqueue");
        if (step > first) ok(mcb200_tallies_collect(ctx, (step - 1) & 1, readback.data()), ctx, "tallies");
      }
      if (step % info.stat_step == info.stat_step - 1) output(step, info.stat_step);
      if (opt.verbose && step % std::max(1, info.stat_step / 10) == 0)
        std::printf("step %d: %zu particles\n", step, mcb200_num_particles(ctx));
    }
    if (opt.readback_every_step && steps > 0)
      ok(mcb200_tallies_collect(ctx, (first + steps - 1) & 1, readback.data()), ctx, "tallies");
    for (int pair = 0; pair < 3; ++pair) settle(pair);
    if (steps > warm) {
      ok(mcb200_mark(ctx, 1), ctx, "mcb200_mark");
      ok(mcb200_elapsed_ms(ctx, 0, 1, &rep->timed_device_ms), ctx, "mcb200_elapsed_ms");
      if (opt.flush_l2_bytes > 0) rep->timed_device_ms = flushed_ms;  // the evictions are not timed
      rep->timed_wall_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - timed_t0).count();
      uint64_t ps1 = 0;
      ok(mcb200_particle_steps(ctx, &ps1), ctx, "mcb200_particle_steps");
      rep->timed_particle_steps = ps1 - ps0;
      rep->timed_steps = steps - warm;
      double tt[6];
      ok(mcb200_get_timing(ctx, tt, 6), ctx, "mcb200_get_timing");
      rep->timed_flight_ms = tt[0];
      rep->timed_flight_launches = (uint64_t)tt[1];
      rep->timed_launches = (uint64_t)tt[5];
    }
    rep->steps_done = steps;
    // heat phase: the last window's mean potential, frozen
    const int hsteps = !info.flag_compute_heat ? 0
                       : (opt.max_heat_steps >= 0 ? std::min(opt.max_heat_steps, info.heat_steps) : info.heat_steps);
    if (hsteps > 0) {
      if (!pot_avg.empty())  // heat_field, src/heat.cpp:100-105
        ok(mcb200_set_potentials(ctx, pot_avg.data(), qc_avg.data()), ctx, "mcb200_set_potentials");
      heat = true;
      ok(mcb200_set_heat_tally(ctx, 1), ctx, "mcb200_set_heat_tally");
      const int window = info.stat_heat_step > 0 ? info.stat_heat_step : info.stat_step;
      ok(mcb200_reset_tallies(ctx), ctx, "mcb200_reset_tallies");
      ok(mcb200_stat_begin(ctx, window), ctx, "mcb200_stat_begin");
      for (int step = 0; step < hsteps; ++step) {
        density(step);
        refresh(step);
        if (step % window == window - 1) output(step, window);
      }
      rep->heat_steps_done = hsteps;
    }
    ok(mcb200_sync(ctx), ctx, "mcb200_sync");
    rep->wall_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    uint64_t ps_end = 0;
    ok(mcb200_particle_steps(ctx, &ps_end), ctx, "mcb200_particle_steps");
    rep->particle_steps = ps_end - ps_start;
    if (info.flag_compute_potential) {
      int64_t solves = 0, its = 0;
      ok(mcb200_poisson_stats(ctx, &solves, &its, &rep->poisson_max_residual, 0), ctx, "mcb200_poisson_stats");
      rep->poisson_solves = (int)solves;
      rep->poisson_iterations = its;
    }
    double tim[6];
    ok(mcb200_get_timing(ctx, tim, 6), ctx, "mcb200_get_timing");
    rep->flight_ms = tim[0];
    rep->step_ms = tim[2];
    rep->final_particles = mcb200_num_particles(ctx);
  }
};

}  // namespace

extern "C" int mcb200_deck_surface_params(const char *input_path, mcb200_ctx *ctx, const mcb200_deck_info *info,
                                          mcb200_surface_params *out, int *poisson_every) {
  if (!input_path || !ctx || !info || !out) return MCB200_ERR_ARG;
  const Extras ex = read_extras(input_path);
  double u[14];
  if (int rc = mcb200_units(ctx, u, 14)) return rc;
  const double spr0 = u[2];
  mcb200_surface_params s{};
  s.delta = ex.delta_nm * 1e-9 / spr0;
  s.ail = ex.lambda_nm * 1e-9 / spr0;
  s.xiph = 12.0; s.theta = 2.857703; s.gama = 1.5; s.nbmod = 2.0;
  s.npf = -0.6; s.pft = 0.7; s.pfn = 0.3; s.kpha = 3600e-4;
  s.roughness = info->flag_surface_roughness;
  s.phonon = info->flag_surface_phonon;
  *out = s;
  if (poisson_every) *poisson_every = ex.poisson_every;
  return MCB200_OK;
}

extern "C" int mcb200_write_outputs(mcb200_ctx *ctx, const char *data_dir, int step, int window, double dt,
                                    int n_contacts, int heat) {
  if (!ctx || !data_dir || window < 1 || n_contacts < 0 || n_contacts > 16 || !(dt > 0)) return MCB200_ERR_ARG;
  mcb200_run_report report{};
  Run r;
  r.ctx = ctx;
  r.rep = &report;
  r.data_dir = data_dir;
  r.heat = heat != 0;
  r.info.dt = dt;
  r.info.n_contacts = n_contacts;
  int rc = MCB200_OK;
  try {
    ok(mcb200_get_mesh_dims(ctx, &r.nx, &r.ny, &r.nz), ctx, "mcb200_get_mesh_dims");
    ok(mcb200_units(ctx, r.u, 14), ctx, "mcb200_units");
    r.cells = r.nx * r.ny * r.nz;
    r.nodes = (r.nx + 1) * (r.ny + 1) * (r.nz + 1);
    r.node_volume.resize(r.nodes);
    ok(mcb200_get_array(ctx, "node_volume", r.node_volume.data(), r.nodes), ctx, "node_volume");
    for (size_t slash = r.data_dir.find('/', 1); slash != std::string::npos; slash = r.data_dir.find('/', slash + 1))
      ::mkdir(r.data_dir.substr(0, slash).c_str(), 0755);  // the parents first (mkdir -p)
    ::mkdir(r.data_dir.c_str(), 0755);
    r.write_outputs(step, window);
  } catch (const RunError &e) {
    rc = e.code ? e.code : MCB200_ERR_STATE;
  } catch (const std::exception &e) {
    rc = MCB200_ERR_IO;
  }
  r.ctx = nullptr;  // the caller's context: not destroyed here
  return rc;
}

extern "C" int mcb200_run_deck(const char *input_path, int device, const mcb200_run_options *options,
                               mcb200_run_report *report, char *error, size_t error_len) {
  if (!input_path || !options || !report) return MCB200_ERR_ARG;
  std::memset(report, 0, sizeof(*report));
  Run r;
  r.opt = *options;
  r.rep = report;
  int rc = MCB200_OK;
  try {
    r.go(input_path, device);
  } catch (const RunError &e) {
    rc = e.code ? e.code : MCB200_ERR_STATE;
    if (error && error_len) std::snprintf(error, error_len, "%s", e.what());
  } catch (const std::exception &e) {
    rc = MCB200_ERR_STATE;
    if (error && error_len) std::snprintf(error, error_len, "%s", e.what());
  }
  if (r.ctx) mcb200_destroy(r.ctx);
  if (r.deck) mcb200_deck_free(r.deck);
  return rc;
}
