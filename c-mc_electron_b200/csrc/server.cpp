// server.cpp -- bias-point requests served by continuous batching
// (mcb200_server_*).  No counterpart in the reference, which runs one bias
// point per process from start to finish.
//
// A request is a device deck (the reference's input.txt / lgrid.txt /
// ldg.txt) plus a family (requests of one family share the mesh, so one can
// warm-start another), its bias, and a completion target for the drain
// current Ids.  Every round the server
//   1. admits queued requests, in arrival order, while a slot is free and
//      its device memory fits the HBM budget (evicting warm-start entries,
//      least recently used first, when that makes room): a context made
//      alike (shared band tables), the deck applied, then either a warm
//      start -- the ensemble and potential of the nearest converged bias of
//      the family, refreshed to this deck's carrier targets -- or the deck's
//      own initial ensemble, and the first Poisson solve;
//   2. runs `quantum` full timesteps of every active request as one batch
//      (mcb200_batch_run: one flight launch per step for all of them, steps
//      replayed from CUDA graphs), so requests admitted while others run
//      overlap with them on the device;
//   3. enqueues the MultipleRefresh of the requests whose refresh step fell
//      in the round, reads every request's contact tallies (one window of
//      Ids per round) and retires the requests whose Ids standard error
//      (windows after the transient, batch means) is below target, or that
//      reached their step limit.  A retired request's context becomes a
//      warm-start entry of its family.
// Every schedule (steps, Poisson solves, refreshes, Ids windows) counts a
// request's own steps from its admission, and every particle draws from its
// own random stream, so a cold-started request gives the same result alone
// or among others.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <deque>
#include <list>
#include <memory>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "mcb200.h"

namespace {

struct Slot;

struct WarmEntry {
  std::string family;
  double bias[2];
  mcb200_ctx *ctx = nullptr;
  size_t bytes = 0;
  uint64_t last_use = 0;
  uint64_t request = 0;
};

struct Slot {
  uint64_t id = 0;
  mcb200_request req{};
  std::string input, family;
  mcb200_ctx *ctx = nullptr;
  mcb200_deck_info info{};
  std::vector<int32_t> refresh_e, refresh_h, eeff;
  mcb200_surface_params surf{};
  int poisson_every = 1;
  uint32_t step = 0;           // the request's own step count
  std::vector<double> windows;  // Ids per window
  int warm = 0;                 // windows still discarded as transient
  uint64_t warm_from = 0;
  size_t bytes = 0;
  double t_admit = 0;
  uint64_t psteps0 = 0;
  double curr0 = 0, time0 = 0;
};

std::string errmsg(mcb200_ctx *c) { return c ? std::string(mcb200_last_error(c)) : std::string("no context"); }

}  // namespace

struct mcb200_server {
  std::string error;
  mcb200_server_options opt{};
  std::string table_dir;
  mcb200_ctx *root = nullptr;  // owns the band tables every request shares
  std::deque<std::unique_ptr<Slot>> pending;
  std::vector<std::unique_ptr<Slot>> active;
  std::list<WarmEntry> cache;
  std::vector<mcb200_result> done;
  mcb200_batch *batch = nullptr;
  bool membership_changed = true;
  uint64_t next_id = 1, rounds = 0, use_counter = 0, retired_particle_steps = 0;
  double device_ms = 0;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();

  double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
  size_t used_bytes() const {
    size_t b = 0;
    for (const auto &s : active) b += s->bytes;
    for (const auto &w : cache) b += w.bytes;
    return b;
  }
  void drop_batch() {
    if (batch) {
      mcb200_batch_sync(batch);
      mcb200_batch_destroy(batch);
      batch = nullptr;
    }
  }
  ~mcb200_server() {
    drop_batch();
    for (auto &s : active)
      if (s->ctx) mcb200_destroy(s->ctx);
    for (auto &w : cache)
      if (w.ctx) mcb200_destroy(w.ctx);
    if (root) mcb200_destroy(root);
  }
};

namespace {

int sfail(mcb200_server *v, int code, const std::string &msg) {
  if (v) v->error = msg;
  return code;
}

size_t free_bytes(int device) {
  size_t f = 0, t = 0;
  cudaSetDevice(device);
  cudaMemGetInfo(&f, &t);
  return f;
}

// Ids of the last window, then the tallies restart.  MCB200_IDS_CONTACT:
// the drain contact's current (the reference's current_scatter_info:
// (CharGen - CharCatch) / (dt * steps) * curr0 * 1e-2).  MCB200_IDS_SECTIONS:
// the net carrier flux through the y node planes (the reference's
// section_current, (rcurrent - lcurrent) / (dt * steps) * curr0 * 1e-2)
// averaged over the middle third of the planes: the same steady-state
// current with far less noise, since every crossing of every plane counts.
// MCB200_IDS_INDUCED: the current the drain carries by induction
// (Ramo-Shockley, summed over every particle at every step): the same
// steady-state current with the least noise, since every particle's motion
// counts, not only its crossings.
int read_window(Slot &s, int steps) {
  std::vector<double> contact(16 * 6), lc(s.info.ny + 1), rc(s.info.ny + 1);
  if (int e = mcb200_get_tallies(s.ctx, nullptr, contact.data(), lc.data(), rc.data(), nullptr, nullptr)) return e;
  double ids = 0;
  if (s.req.ids_estimator == MCB200_IDS_INDUCED) {
    double sum = 0, n = 0;
    if (int e = mcb200_get_induced_current(s.ctx, &sum, &n)) return e;
    ids = n > 0 ? sum / n * s.curr0 * 1e-2 : 0.0;
  } else if (s.req.ids_estimator == MCB200_IDS_SECTIONS) {
    const int ny = s.info.ny, j0 = ny / 3, j1 = std::max(j0 + 1, ny - ny / 3);
    for (int j = j0; j < j1; ++j) ids += rc[j] - lc[j];
    ids = ids / (j1 - j0) / (s.info.dt * steps) * s.curr0 * 1e-2;
  } else {
    const int c = std::min(std::max(s.req.drain_contact, 0), 15);
    ids = (contact[6 * c + 1] - contact[6 * c + 4]) / (s.info.dt * steps) * s.curr0 * 1e-2;
  }
  if (s.warm > 0) --s.warm;
  else s.windows.push_back(ids);
  return mcb200_reset_tallies(s.ctx);
}

// Batch means: mean Ids and its standard error over the kept windows.
void ids_stats(const Slot &s, double &mean, double &stderr_) {
  const size_t n = s.windows.size();
  mean = 0;
  for (double v : s.windows) mean += v;
  mean = n ? mean / n : 0.0;
  double var = 0;
  for (double v : s.windows) var += (v - mean) * (v - mean);
  stderr_ = n > 1 ? std::sqrt(var / (n - 1) / n) : INFINITY;
}

// Everything an admitted request needs before its first step.
int admit(mcb200_server *v, Slot &s) {
  mcb200_deck *deck = nullptr;
  auto deck_err = [&](int rc, const char *what) {
    const std::string m = std::string(what) + ": " + (deck ? mcb200_deck_error(deck) : "");
    if (deck) mcb200_deck_free(deck);
    return sfail(v, rc, m);
  };
  if (int rc = mcb200_deck_load(s.input.c_str(), &deck)) return deck_err(rc, "mcb200_deck_load");
  if (int rc = mcb200_deck_prepare(deck, v->root)) return deck_err(rc, "mcb200_deck_prepare");
  mcb200_deck_get_info(deck, &s.info);
  auto ints = [&](const char *name, std::vector<int32_t> &out) {
    size_t n = 0;
    mcb200_deck_int_array(deck, name, nullptr, 0, &n);
    out.resize(n);
    return mcb200_deck_int_array(deck, name, out.data(), n, &n);
  };
  std::vector<int32_t> en, hn;
  if (ints("electron_num", en) || ints("hole_num", hn) || ints("refresh_electrons", s.refresh_e) ||
      ints("refresh_holes", s.refresh_h) || ints("eeff_direction", s.eeff))
    return deck_err(MCB200_ERR_STATE, "deck arrays");
  size_t start = 0, target = 0;
  for (size_t c = 0; c < en.size(); ++c) {
    start += (size_t)en[c] + hn[c];
    target += (size_t)s.refresh_e[c] + s.refresh_h[c];
  }
  // a warm start: the nearest converged bias of the family; with
  // MCB200_WARM_SETTLED, failing that, the nearest running request of the
  // family past its transient (its ensemble as the last round left it)
  WarmEntry *from = nullptr;
  const Slot *from_slot = nullptr;
  if (s.req.warm_start) {
    double best = INFINITY;
    for (auto &w : v->cache) {
      if (w.family != s.family) continue;
      const double d = std::hypot(w.bias[0] - s.req.bias[0], w.bias[1] - s.req.bias[1]);
      if (d < best) {
        best = d;
        from = &w;
      }
    }
  }
  if (!from && s.req.warm_start == MCB200_WARM_SETTLED) {
    double best = INFINITY;
    for (const auto &a : v->active) {
      if (a->family != s.family || a->warm > 0 || a->windows.empty()) continue;
      const double d = std::hypot(a->req.bias[0] - s.req.bias[0], a->req.bias[1] - s.req.bias[1]);
      if (d < best) {
        best = d;
        from_slot = a.get();
      }
    }
  }
  mcb200_ctx *donor = from ? from->ctx : (from_slot ? from_slot->ctx : nullptr);
  size_t from_n = 0;
  if (donor) from_n = mcb200_num_particles(donor);
  const size_t big = std::max(std::max(start, target), from_n);
  const size_t capacity = big + big / 4 + 65536;
  const size_t before = free_bytes(v->opt.device);
  if (int rc = mcb200_create_alike(v->root, capacity, &s.ctx)) {
    const std::string m = errmsg(s.ctx);
    mcb200_deck_free(deck);
    return sfail(v, rc, "mcb200_create_alike: " + m);
  }
  auto ctx_err = [&](int rc, const char *what) {
    const std::string m = std::string(what) + ": " + errmsg(s.ctx);
    if (deck) mcb200_deck_free(deck);
    deck = nullptr;
    return sfail(v, rc, m);
  };
  if (v->opt.flight_precision)
    if (int rc = mcb200_set_flight_precision(s.ctx, v->opt.flight_precision)) return ctx_err(rc, "precision");
  double u[14];
  mcb200_units(s.ctx, u, 14);
  s.curr0 = u[12];
  s.time0 = u[3];
  if (int rc = mcb200_apply_deck(s.ctx, deck)) return deck_err(rc, "mcb200_apply_deck");
  int pe = 1;
  if (int rc = mcb200_deck_surface_params(s.input.c_str(), s.ctx, &s.info, &s.surf, &pe))
    return ctx_err(rc, "surface parameters");
  s.poisson_every = s.req.poisson_every > 0 ? s.req.poisson_every : pe;
  // the refresh targets go to the device now, not at the first refresh inside a running batch
  if (int rc = mcb200_set_refresh_targets(s.ctx, s.refresh_e.data(), s.refresh_h.data()))
    return ctx_err(rc, "mcb200_set_refresh_targets");
  if (donor) {
    if (int rc = mcb200_copy_ensemble(s.ctx, donor)) return ctx_err(rc, "mcb200_copy_ensemble");
    // to this deck's carrier targets, as a refresh would
    if (int rc = mcb200_multiple_refresh(s.ctx, s.refresh_e.data(), s.refresh_h.data(), 0, s.req.seed, nullptr))
      return ctx_err(rc, "warm-start refresh");
    if (from) {
      from->last_use = ++v->use_counter;
      s.warm_from = from->request;
    } else {
      s.warm_from = from_slot->id;
    }
    s.warm = s.req.warm_windows_warm;
  } else {
    if (int rc = mcb200_seed_deck(s.ctx, deck, s.req.seed)) return deck_err(rc, "mcb200_seed_deck");
    s.warm = s.req.warm_windows_cold;
  }
  mcb200_deck_free(deck);
  deck = nullptr;  // the error paths below must not free it again
  if (int rc = mcb200_deposit(s.ctx)) return ctx_err(rc, "mcb200_deposit");
  if (s.info.flag_compute_potential) {
    int it = 0;
    double res = 0;
    if (int rc = mcb200_solve_poisson(s.ctx, 1e-10, 20000, &it, &res)) return ctx_err(rc, "first Poisson solve");
  }
  if (s.info.flag_surface_scatter)
    if (int rc = mcb200_surface_rates(s.ctx, &s.surf, s.eeff.data())) return ctx_err(rc, "surface rates");
  if (s.req.ids_estimator == MCB200_IDS_INDUCED)
    if (int rc = mcb200_set_induced_current(s.ctx, std::min(std::max(s.req.drain_contact, 0), 15)))
      return ctx_err(rc, "weighting field");
  mcb200_reset_tallies(s.ctx);
  mcb200_sync(s.ctx);
  mcb200_particle_steps(s.ctx, &s.psteps0);
  const size_t after = free_bytes(v->opt.device);
  s.bytes = before > after ? before - after : 0;
  s.t_admit = v->now();
  return MCB200_OK;
}

// Room for `need` more bytes: least recently used warm-start entries go first.
bool make_room(mcb200_server *v, size_t need) {
  const size_t budget = v->opt.hbm_budget_bytes;
  while (v->used_bytes() + need > budget && !v->cache.empty()) {
    auto lru = std::min_element(v->cache.begin(), v->cache.end(),
                                [](const WarmEntry &a, const WarmEntry &b) { return a.last_use < b.last_use; });
    mcb200_destroy(lru->ctx);
    v->cache.erase(lru);
  }
  return v->used_bytes() + need <= budget;
}

// The device memory a request will take: what an admitted request of its
// family took.  The first request of a family is admitted on trust and
// measured (cudaMemGetInfo around its set-up); if it overshoots the budget,
// warm-start entries are evicted and later admissions wait.
size_t estimate_bytes(const mcb200_server *v, const Slot &s) {
  for (const auto &a : v->active)
    if (a->family == s.family) return a->bytes;
  for (const auto &w : v->cache)
    if (w.family == s.family) return w.bytes;
  return 0;
}

void retire(mcb200_server *v, size_t k, int status) {
  Slot &s = *v->active[k];
  mcb200_result r{};
  r.id = s.id;
  r.status = status;
  ids_stats(s, r.ids, r.ids_stderr);
  r.windows = (int)s.windows.size();
  r.steps = (int)s.step;
  uint64_t ps = 0;
  mcb200_particle_steps(s.ctx, &ps);
  r.particle_steps = ps - s.psteps0;
  v->retired_particle_steps += r.particle_steps;
  r.arrival_s = s.req.arrival_s;
  r.admit_s = s.t_admit;
  r.done_s = v->now();
  r.warm_from = s.warm_from;
  r.particles = mcb200_num_particles(s.ctx);
  r.bytes = s.bytes;
  v->done.push_back(r);
  if (status == MCB200_SERVE_CONVERGED && s.req.warm_start) {
    WarmEntry w;
    w.family = s.family;
    w.bias[0] = s.req.bias[0];
    w.bias[1] = s.req.bias[1];
    w.ctx = s.ctx;
    w.bytes = s.bytes;
    w.last_use = ++v->use_counter;
    w.request = s.id;
    v->cache.push_back(w);
  } else {
    mcb200_destroy(s.ctx);
  }
  s.ctx = nullptr;
  v->active.erase(v->active.begin() + (long)k);
  v->membership_changed = true;
}

}  // namespace

extern "C" {

int mcb200_server_create(const mcb200_server_options *opt, mcb200_server **out) {
  if (!opt || !out || !opt->table_dir) return MCB200_ERR_ARG;
  mcb200_server *v = new mcb200_server;
  *out = v;
  v->opt = *opt;
  v->table_dir = opt->table_dir;
  v->opt.table_dir = v->table_dir.c_str();
  if (v->opt.hbm_budget_bytes == 0) v->opt.hbm_budget_bytes = (size_t)160 << 30;
  if (v->opt.max_slots <= 0 || v->opt.max_slots > 64) v->opt.max_slots = 64;
  if (v->opt.quantum_steps <= 0) v->opt.quantum_steps = 50;
  if (int rc = mcb200_create(v->opt.table_dir, opt->kelvin > 0 ? opt->kelvin : 300.0, opt->device, 1, &v->root))
    return sfail(v, rc, "band tables: " + errmsg(v->root));
  return MCB200_OK;
}

void mcb200_server_destroy(mcb200_server *v) { delete v; }

const char *mcb200_server_last_error(const mcb200_server *v) { return v ? v->error.c_str() : "null server"; }

double mcb200_server_now(const mcb200_server *v) { return v ? v->now() : 0.0; }

int mcb200_server_submit(mcb200_server *v, const mcb200_request *req, uint64_t *id) {
  if (!v || !req || !req->input_path || !req->family) return MCB200_ERR_ARG;
  if (req->warm_start < MCB200_WARM_OFF || req->warm_start > MCB200_WARM_SETTLED) return MCB200_ERR_ARG;
  auto s = std::make_unique<Slot>();
  s->id = v->next_id++;
  s->req = *req;
  s->input = req->input_path;
  s->family = req->family;
  s->req.input_path = s->input.c_str();
  s->req.family = s->family.c_str();
  if (s->req.target_rel_err <= 0) s->req.target_rel_err = 0.01;
  if (s->req.min_windows < 2) s->req.min_windows = 2;
  if (id) *id = s->id;
  v->pending.push_back(std::move(s));
  return MCB200_OK;
}

int mcb200_server_round(mcb200_server *v, int *active, int *pending) {
  if (!v) return MCB200_ERR_ARG;
  const int q = v->opt.quantum_steps;
  // 1. admissions, in arrival order
  while (!v->pending.empty() && (int)v->active.size() < v->opt.max_slots) {
    Slot &s = *v->pending.front();
    if (!make_room(v, estimate_bytes(v, s))) break;  // the head waits for memory; so do the others
    v->drop_batch();
    if (int rc = admit(v, s)) {
      mcb200_result r{};
      r.id = s.id;
      r.status = rc < 0 ? rc : -rc;
      r.arrival_s = s.req.arrival_s;
      r.done_s = v->now();
      v->done.push_back(r);
      if (s.ctx) mcb200_destroy(s.ctx);
      v->pending.pop_front();
      continue;
    }
    v->active.push_back(std::move(v->pending.front()));
    v->pending.pop_front();
    v->membership_changed = true;
    if (v->used_bytes() > v->opt.hbm_budget_bytes) make_room(v, 0);
  }
  if (!v->active.empty()) {
    // 2. one quantum of every active request, as one batch
    if (v->membership_changed || !v->batch) {
      v->drop_batch();
      std::vector<mcb200_ctx *> ctxs;
      std::vector<mcb200_batch_member> m;
      for (auto &s : v->active) {
        ctxs.push_back(s->ctx);
        mcb200_batch_member b{};
        b.dt = s->info.dt;
        b.seed = s->req.seed;
        b.first_step = s->step;
        b.self_consistent = s->info.flag_compute_potential;
        b.poisson_every = s->poisson_every;
        b.surface_rates = s->info.flag_surface_scatter;
        m.push_back(b);
      }
      if (int rc = mcb200_batch_create(ctxs.data(), m.data(), (int)ctxs.size(), &v->batch)) {
        const std::string e = v->batch ? mcb200_batch_last_error(v->batch) : "";
        if (v->batch) mcb200_batch_destroy(v->batch);
        v->batch = nullptr;
        return sfail(v, rc, "mcb200_batch_create: " + e);
      }
      mcb200_batch_use_graphs(v->batch, v->opt.use_graphs);
      v->membership_changed = false;
    }
    mcb200_batch_mark(v->batch, 0);
    if (int rc = mcb200_batch_run(v->batch, q)) return sfail(v, rc, std::string("mcb200_batch_run: ") +
                                                                        mcb200_batch_last_error(v->batch));
    for (auto &s : v->active) {
      const uint32_t first = s->step;
      s->step += (uint32_t)q;
      // 3. refreshes whose step fell in the round (the reference's step % mr_step == mr_step - 1)
      if (s->info.flag_multiple_refresh && s->info.mr_step > 0) {
        int64_t hit = -1;
        for (uint32_t t = first; t < s->step; ++t)
          if ((int)(t % (uint32_t)s->info.mr_step) == s->info.mr_step - 1) hit = t;
        if (hit >= 0)
          mcb200_multiple_refresh(s->ctx, s->refresh_e.data(), s->refresh_h.data(), (uint32_t)hit, s->req.seed,
                                  nullptr);
      }
    }
    mcb200_batch_mark(v->batch, 1);
    double ms = 0;
    mcb200_batch_elapsed_ms(v->batch, 0, 1, &ms);  // waits for the round
    v->device_ms += ms;
    ++v->rounds;
    std::vector<int> verdict(v->active.size(), 0);
    bool any = false;
    for (size_t k = 0; k < v->active.size(); ++k) {
      Slot &s = *v->active[k];
      if (int rc = read_window(s, q)) return sfail(v, rc, "tallies: " + errmsg(s.ctx));
      double mean = 0, se = 0;
      ids_stats(s, mean, se);
      const bool enough = (int)s.windows.size() >= s.req.min_windows;
      if (enough && std::fabs(se) <= s.req.target_rel_err * std::fabs(mean) && mean != 0.0)
        verdict[k] = MCB200_SERVE_CONVERGED;
      else if (s.req.max_steps > 0 && (int)s.step >= s.req.max_steps)
        verdict[k] = MCB200_SERVE_STEP_LIMIT;
      any = any || verdict[k] != 0;
    }
    if (any) {
      // the batch holds the members' contexts: it goes before any of them is
      // destroyed or cached (the round's work is complete: its end mark was waited for)
      mcb200_batch_destroy(v->batch);
      v->batch = nullptr;
      for (size_t k = v->active.size(); k-- > 0;)
        if (verdict[k]) retire(v, k, verdict[k]);
    }
  }
  if (active) *active = (int)v->active.size();
  if (pending) *pending = (int)v->pending.size();
  return MCB200_OK;
}

int mcb200_server_results(mcb200_server *v, mcb200_result *out, int max, int *n) {
  if (!v || !n || (max > 0 && !out)) return MCB200_ERR_ARG;
  const int k = std::min<int>(max, (int)v->done.size());
  for (int i = 0; i < k; ++i) out[i] = v->done[i];
  v->done.erase(v->done.begin(), v->done.begin() + k);
  *n = k;
  return MCB200_OK;
}

int mcb200_server_stats(const mcb200_server *v, mcb200_server_stats_t *st) {
  if (!v || !st) return MCB200_ERR_ARG;
  st->rounds = v->rounds;
  st->device_ms = v->device_ms;
  uint64_t ps = v->retired_particle_steps;
  for (const auto &s : v->active) {
    uint64_t p = 0;
    mcb200_particle_steps(s->ctx, &p);
    ps += p - s->psteps0;
  }
  st->particle_steps = ps;
  st->active = (int)v->active.size();
  st->pending = (int)v->pending.size();
  st->cached = (int)v->cache.size();
  st->bytes_in_use = v->used_bytes();
  return MCB200_OK;
}

}  // extern "C"
