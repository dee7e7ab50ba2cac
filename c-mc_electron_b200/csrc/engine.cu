// engine.cu -- context, device-table upload and the C ABI of include/mcb200.h.
#include <algorithm>
#include <list>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "engine_internal.h"

#include <mutex>

using namespace mcb200;
using namespace mcb200::eng;

namespace mcb200::eng {

int fail(mcb200_ctx *c, int code, const std::string &msg) {
  if (c) c->error = msg;
  return code;
}

// After a refresh: the particle count is the emitted total, the uid counter
// advances past the new particles (tot = {emitted, new uids}).
__global__ void refresh_counts_kernel(unsigned int *d, const unsigned int *tot) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    d[0] = tot[0];
    d[1] += tot[1];
  }
}

__global__ void set_counts_kernel(unsigned int *d, unsigned int n, unsigned int next_uid) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    d[0] = n;
    d[1] = next_uid;
  }
}

// Host copies of the device counts, after the stream has drained (only when
// a step may have changed them).  A store-full flag raised by a step is
// reported here, once.
void pull_counts(mcb200_ctx *c) {
  if (c->n_stale) {
    ck(cudaMemcpyAsync(c->h_pinned + 32, c->dev_counts, 3 * sizeof(unsigned int), cudaMemcpyDeviceToHost, c->stream),
       "count");
    ck(cudaStreamSynchronize(c->stream), "sync");
    c->n = c->h_pinned[32];
    c->next_uid = c->h_pinned[33];
    c->n_stale = false;
    if (c->h_pinned[34]) {
      ck(cudaMemsetAsync(c->dev_counts + 2, 0, sizeof(unsigned int), c->stream), "memset");
      c->overflow_pending = true;
    }
  }
  if (c->overflow_pending) {
    c->overflow_pending = false;
    throw CapacityError("particle store full: GENERATE copies beyond the context capacity were dropped");
  }
}

// The host's counts into device memory (after the host changed the store).
void push_counts(mcb200_ctx *c) {
  set_counts_kernel<<<1, 32, 0, c->stream>>>(c->dev_counts, (unsigned int)c->n, c->next_uid);
  ck(cudaGetLastError(), "set counts");
  c->n_stale = false;
}

// Reads back the timing of ring slot q (its events are complete or the call waits for them).
void harvest_timing(mcb200_ctx *c, int q) {
  if (!c->ev_pending[q]) return;
  ck(cudaEventSynchronize(c->ev[q][3]), "cudaEventSynchronize");
  float ms_flight = 0, ms_step = 0;
  ck(cudaEventElapsedTime(&ms_flight, c->ev[q][1], c->ev[q][2]), "elapsed");
  ck(cudaEventElapsedTime(&ms_step, c->ev[q][0], c->ev[q][3]), "elapsed");
  c->flight_ms += ms_flight;
  c->step_ms += ms_step;
  c->ev_pending[q] = false;
}
void harvest_all_timing(mcb200_ctx *c) {
  for (int q = 0; q < mcb200_ctx::kTimingRing; ++q) harvest_timing(c, q);
}


// Particle and child buffers for the context's precision.
void alloc_stores(mcb200_ctx *c) {
  for (void *p : c->store_owned) cudaFree(p);
  c->store_owned.clear();
  for (int i = 0; i < 2; ++i) c->pb[i] = ParticleBuffers{};
  for (int g = 0; g < mcb200_ctx::kGenerations; ++g) c->cb[g] = ChildBuffers{};
  for (int i = 0; i < 2; ++i) {
    if (c->precision == MCB200_FLIGHT_FP32) alloc_particles(c->pb[i].f, c->capacity, c->store_owned);
    else alloc_particles(c->pb[i].d, c->capacity, c->store_owned);
  }
  for (int g = 0; g < mcb200_ctx::kGenerations; ++g) {
    if (c->precision == MCB200_FLIGHT_FP32) alloc_children(c->cb[g].f, c->child_cap, c->store_owned);
    else alloc_children(c->cb[g].d, c->child_cap, c->store_owned);
  }
}

// The charge bounds of the current store (its device count) into c->bounds,
// on the context's stream.  Every path that writes the store calls it after
// writing, except the step, whose sort computes them.
void store_bounds(mcb200_ctx *c) {
  const DevCount n{c->dev_counts, nullptr, (int)c->capacity};
  const int grid = grid_for(c, c->capacity, 256);
  if (c->precision == MCB200_FLIGHT_FP32) launch_charge_bounds(store<float>(c, c->cur), n, c->bounds, grid, c->stream);
  else launch_charge_bounds(store<double>(c, c->cur), n, c->bounds, grid, c->stream);
  ck(cudaGetLastError(), "charge bounds");
}

// Uniform k-space locator for the tetrahedron search (see flight_physics.cuh).
void build_kgrid(mcb200_ctx *c, int g) {
  const FullBandTables &t = c->ts->tab;
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int i = 0; i < t.nk; ++i) {
    const double v[3] = {t.xkk[i], t.ykk[i], t.zkk[i]};
    for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], v[a]); hi[a] = std::max(hi[a], v[a]); }
  }
  const double pad = 1e-9 * t.u.a0pi;
  for (int a = 0; a < 3; ++a) { lo[a] -= pad; hi[a] += pad; }
  double inv[3];
  for (int a = 0; a < 3; ++a) inv[a] = g / (hi[a] - lo[a]);
  const int cells = g * g * g;
  std::vector<std::vector<int>> lists((size_t)kMNB * cells);
  for (int it = t.nt - 1; it >= 0; --it) {  // descending tet order inside each cell
    double blo[3] = {1e300, 1e300, 1e300}, bhi[3] = {-1e300, -1e300, -1e300};
    for (int v = 0; v < 4; ++v) {
      const int nd = t.T(v, it);
      const double p[3] = {t.xkk[nd], t.ykk[nd], t.zkk[nd]};
      for (int a = 0; a < 3; ++a) { blo[a] = std::min(blo[a], p[a]); bhi[a] = std::max(bhi[a], p[a]); }
    }
    int c0[3], c1[3];
    for (int a = 0; a < 3; ++a) {
      c0[a] = std::max(0, std::min(g - 1, (int)std::floor((blo[a] - pad - lo[a]) * inv[a])));
      c1[a] = std::max(0, std::min(g - 1, (int)std::floor((bhi[a] + pad - lo[a]) * inv[a])));
    }
    for (int i = c0[0]; i <= c1[0]; ++i)
      for (int j = c0[1]; j <= c1[1]; ++j)
        for (int k = c0[2]; k <= c1[2]; ++k) lists[(size_t)t.ibt[it] * cells + (i * g + j) * g + k].push_back(it);
  }
  std::vector<int> start((size_t)kMNB * (cells + 1)), tets;
  for (int b = 0; b < kMNB; ++b) {
    int *st = &start[(size_t)b * (cells + 1)];
    for (int q = 0; q < cells; ++q) {
      st[q] = (int)tets.size();
      const auto &l = lists[(size_t)b * cells + q];
      tets.insert(tets.end(), l.begin(), l.end());
    }
    st[cells] = (int)tets.size();
  }
  c->ts->dt.grid_n = g;
  for (int a = 0; a < 3; ++a) { c->ts->dt.grid_lo[a] = lo[a]; c->ts->dt.grid_inv[a] = inv[a]; }
  c->ts->dt.grid_start = dupload(start, c->ts->owned);
  c->ts->dt.grid_tets = dupload(tets, c->ts->owned);

  // Seed grid for the lowest conduction band (the band impurity scattering
  // lands in): per fine cell, a tetrahedron that contains the cell centre,
  // else the first tetrahedron overlapping it, else -1.  A mesh walk from
  // the seed reaches the target point in a step or two.
  const int sg = kSeedGridN;
  std::vector<int> seed((size_t)sg * sg * sg, -1);
  const int band = t.bandof[0];
  const int *bst = &start[(size_t)band * (cells + 1)];
  auto contains = [&](int it, double a, double b, double cc) {
    for (int f = 0; f < 4; ++f)
      if (t.D(0, f, it) * a + t.D(1, f, it) * b + t.D(2, f, it) * cc - t.D(3, f, it) < -1e-13) return false;
    return true;
  };
  for (int i = 0; i < sg; ++i)
    for (int j = 0; j < sg; ++j)
      for (int k = 0; k < sg; ++k) {
        const double p[3] = {lo[0] + (i + 0.5) * (hi[0] - lo[0]) / sg, lo[1] + (j + 0.5) * (hi[1] - lo[1]) / sg,
                             lo[2] + (k + 0.5) * (hi[2] - lo[2]) / sg};
        int q[3];
        for (int a = 0; a < 3; ++a) q[a] = std::max(0, std::min(g - 1, (int)std::floor((p[a] - lo[a]) * inv[a])));
        const int coarse = (q[0] * g + q[1]) * g + q[2];
        int pick = -1;
        for (int e = bst[coarse]; e < bst[coarse + 1]; ++e) {
          const int it = tets[e];
          if (pick < 0) pick = it;
          if (contains(it, p[0], p[1], p[2])) {
            pick = it;
            break;
          }
        }
        seed[((size_t)i * sg + j) * sg + k] = pick;
      }
  for (int a = 0; a < 3; ++a) c->ts->dt.seed_inv[a] = sg / (hi[a] - lo[a]);
  c->ts->dt.seed_grid = dupload(seed, c->ts->owned);
}

template <typename T>
std::vector<float> to_float(const std::vector<T> &v) {
  return std::vector<float>(v.begin(), v.end());
}

// FP32 copies of the flight tables.  Face planes are scaled to unit normals
// (the sign of every face test and every drift-time ratio is unchanged), so
// the FP32 containment tolerance is a k-space distance.
void upload_tables32(mcb200_ctx *c, const std::vector<TetFlight> &tf, const std::vector<TetShape> &ts,
                     const std::vector<double4> &kn) {
  const FullBandTables &t = c->ts->tab;
  DevTables32 &d = c->ts->dt.f32;
  std::vector<TetFlightT<float>> tf32(tf.size(), TetFlightT<float>{});
  std::vector<TetShapeT<float>> ts32(ts.size());
  for (size_t it = 0; it < tf.size(); ++it) {
    for (int f = 0; f < 4; ++f) {
      const double *n = tf[it].n[f];
      const double len = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
      const double sc = len > 0 ? 1.0 / len : 1.0;
      for (int cc = 0; cc < 4; ++cc) tf32[it].n[f][cc] = (float)(n[cc] * sc);
    }
    for (int cc = 0; cc < 4; ++cc) tf32[it].v[cc] = (float)tf[it].v[cc];
    for (int f = 0; f < 4; ++f) tf32[it].neib[f] = tf[it].neib[f];
    tf32[it].gam = (float)tf[it].gam;
    tf32[it].e0 = (float)tf[it].e0;
    tf32[it].e3 = (float)tf[it].e3;
    tf32[it].band = tf[it].band;
    tf32[it].node0 = tf[it].node0;
    for (int v = 0; v < 4; ++v) ts32[it].e[v] = (float)ts[it].e[v];
    for (int v = 0; v < 3; ++v) ts32[it].fac[v] = (float)ts[it].fac[v];
    ts32[it].vgt = (float)ts[it].vgt;
  }
  std::vector<float4> kn32(kn.size());
  for (size_t i = 0; i < kn.size(); ++i)
    kn32[i] = make_float4((float)kn[i].x, (float)kn[i].y, (float)kn[i].z, (float)kn[i].w);
  d.tf = dupload(tf32, c->ts->owned);
  d.ts = dupload(ts32, c->ts->owned);
  d.knode = dupload(kn32, c->ts->owned);
  d.gamtet = dupload(to_float(t.gamtet), c->ts->owned);
  d.energy = dupload(to_float(t.energy), c->ts->owned);
  d.sumscatt = dupload(to_float(t.sumscatt), c->ts->owned);
  d.scatte = dupload(to_float(t.scatte), c->ts->owned);
  d.dose = dupload(to_float(t.dose), c->ts->owned);
  d.scattiie = dupload(to_float(t.scattiie), c->ts->owned);
  d.scatth = dupload(to_float(t.scatth), c->ts->owned);
  d.dosh = dupload(to_float(t.dosh), c->ts->owned);
  d.scattiih = dupload(to_float(t.scattiih), c->ts->owned);
  d.dostetmax = dupload(to_float(t.dostetmax), c->ts->owned);
}

void upload_tables(mcb200_ctx *c) {
  const FullBandTables &t = c->ts->tab;
  DevTables &d = c->ts->dt;
  d.nt = t.nt; d.nk = t.nk; d.nbt = t.nbt;
  for (int i = 0; i < 3; ++i) { d.nband[i] = t.nband[i]; d.bandof[i] = t.bandof[i]; d.difpr[i] = t.difpr[i]; }
  d.scpre = t.scpre; d.scprh = t.scprh;
  d.dtable = t.dtable; d.emax = t.emax; d.dlist = t.dlist; d.dlists = t.dlists;
  d.temptag = t.temptag; d.templag = t.templag; d.templog = t.templog;
  d.temptaf = t.temptaf; d.templaf = t.templaf; d.temptof = t.temptof; d.temphop = t.temphop;
  d.mell = t.mell; d.melt = t.melt; d.meld = t.meld;
  d.a0pi = t.u.a0pi; d.sieg = t.u.sieg; d.eV0 = t.u.eV0; d.conc0 = t.u.conc0; d.scrt0 = t.u.scrt0;
  d.eps_si = t.u.eps_silicon; d.frickel = t.u.frickel;
  std::vector<TetFlight> tf(t.nt, TetFlight{});
  std::vector<TetShape> ts(t.nt);
  std::vector<int4> tn(t.nt), tb(t.nt);
  for (int it = 0; it < t.nt; ++it) {
    for (int f = 0; f < 4; ++f)
      for (int cc = 0; cc < 4; ++cc) tf[it].n[f][cc] = t.D(cc, f, it);
    for (int cc = 0; cc < 4; ++cc) tf[it].v[cc] = t.vt[(size_t)4 * it + cc];
    for (int f = 0; f < 4; ++f) tf[it].neib[f] = t.N(f, it);
    tf[it].gam = t.gamtet[it];
    tf[it].e0 = t.eek[t.T(0, it)];
    tf[it].e3 = t.eek[t.T(3, it)];
    tf[it].band = t.ibt[it];
    tf[it].node0 = t.T(0, it);
    for (int v = 0; v < 4; ++v) ts[it].e[v] = t.eek[t.T(v, it)];
    ts[it].fac[0] = t.faclow[it]; ts[it].fac[1] = t.facmedium[it]; ts[it].fac[2] = t.fachigh[it];
    ts[it].vgt = t.vgt[it];
    tn[it] = make_int4(t.T(0, it), t.T(1, it), t.T(2, it), t.T(3, it));
    tb[it] = make_int4(t.N(0, it), t.N(1, it), t.N(2, it), t.N(3, it));
  }
  d.tf = dupload(tf, c->ts->owned);
  d.ts = dupload(ts, c->ts->owned);
  d.tnode = dupload(tn, c->ts->owned);
  d.tneib = dupload(tb, c->ts->owned);
  d.ibt = dupload(t.ibt, c->ts->owned);
  d.gamtet = dupload(t.gamtet, c->ts->owned);
  std::vector<double4> kn(t.nk);
  for (int i = 0; i < t.nk; ++i) kn[i] = make_double4(t.xkk[i], t.ykk[i], t.zkk[i], t.eek[i]);
  d.knode = dupload(kn, c->ts->owned);
  d.energy = dupload(t.energy, c->ts->owned);
  d.sumscatt = dupload(t.sumscatt, c->ts->owned);
  d.scatte = dupload(t.scatte, c->ts->owned);
  d.dose = dupload(t.dose, c->ts->owned);
  d.scattiie = dupload(t.scattiie, c->ts->owned);
  d.scatth = dupload(t.scatth, c->ts->owned);
  d.dosh = dupload(t.dosh, c->ts->owned);
  d.scattiih = dupload(t.scattiih, c->ts->owned);
  d.dostetmax = dupload(t.dostetmax, c->ts->owned);
  d.dos = dupload(t.dos, c->ts->owned);
  d.sumdos = dupload(t.sumdos, c->ts->owned);
  for (int i = 0; i < 3; ++i) d.dosmax[i] = t.dosmax[i];
  d.ntlist = dupload(t.ntlist, c->ts->owned); d.ptlist = dupload(t.ptlist, c->ts->owned); d.tlist = dupload(t.tlist, c->ts->owned);
  d.nslist = dupload(t.nslist, c->ts->owned); d.pslist = dupload(t.pslist, c->ts->owned); d.slist = dupload(t.slist, c->ts->owned);
  d.ntlists = dupload(t.ntlists, c->ts->owned); d.ptlists = dupload(t.ptlists, c->ts->owned); d.tlists = dupload(t.tlists, c->ts->owned);
  std::vector<int> symi(48 * 6), newisym(5 * 48), indmat(t.indmat, t.indmat + 729), refl(3 * 48);
  std::vector<double> bz(3 * 5 * 48);
  for (int s = 0; s < 48; ++s)
    for (int cc = 0; cc < 6; ++cc) symi[s * 6 + cc] = t.matsym[cc][s];
  for (int iv = 0; iv < 5; ++iv)
    for (int s = 0; s < 48; ++s) {
      newisym[iv * 48 + s] = t.newisym[iv][s];
      bz[(0 * 5 + iv) * 48 + s] = t.xbz[iv][s];
      bz[(1 * 5 + iv) * 48 + s] = t.ybz[iv][s];
      bz[(2 * 5 + iv) * 48 + s] = t.zbz[iv][s];
    }
  // Reflect / Diffuse mirror tables: isym after negating k_x, k_y or k_z
  // (src/CellHit.cpp:217-238, the indmat lookups with one sign flipped).
  for (int axis = 0; axis < 3; ++axis)
    for (int s = 0; s < 48; ++s) {
      int sg[3] = {t.matsym[3][s], t.matsym[4][s], t.matsym[5][s]};
      sg[axis] = -sg[axis];
      const int idx = (((((sg[0] + 1) * 3 + (sg[1] + 1)) * 3 + (sg[2] + 1)) * 3 + (t.matsym[0][s] - 1)) * 3 +
                       (t.matsym[1][s] - 1)) * 3 + (t.matsym[2][s] - 1);
      refl[axis * 48 + s] = t.indmat[idx];
    }
  d.symi = dupload(symi, c->ts->owned);
  d.newisym = dupload(newisym, c->ts->owned);
  d.bz = dupload(bz, c->ts->owned);
  d.indmat = dupload(indmat, c->ts->owned);
  d.reflect_isym = dupload(refl, c->ts->owned);
  d.disp = t.dispersion.empty() ? nullptr : dupload(t.dispersion, c->ts->owned);
  for (int i = 0; i < kDispTables; ++i) d.disp_off[i] = t.disp_off[i];
  build_kgrid(c, 40);
  upload_tables32(c, tf, ts, kn);
  c->ts->vmax = 0;
  for (size_t q = 0; q < t.vt.size(); ++q)
    if (q % 4 != 3) c->ts->vmax = std::max(c->ts->vmax, std::fabs(t.vt[q]));
}

template <typename T>
void copy_vec(const std::vector<T> &v, void *out, size_t bytes, size_t *needed) {
  *needed = v.size() * sizeof(T);
  if (out && bytes >= *needed) std::memcpy(out, v.data(), *needed);
}

int grid_for(const mcb200_ctx *c, size_t n, int block) {
  const size_t want = (n + block - 1) / block;
  const size_t cap = (size_t)c->sm_count * (size_t)c->grid_per_sm;
  return (int)std::max<size_t>(1, std::min(want, cap));
}

// MgHierarchy::build for the node grid, stencil and Dirichlet pattern, from
// a small process-wide cache: the hierarchy depends on nothing else, so the
// contexts of one device shape at other biases (a bias sweep, the members of
// a batch, served requests) share one host build.  Entries hold their
// inputs and match them exactly.  Null when the mesh does not coarsen.
std::shared_ptr<const MgHierarchy> cached_hierarchy(int px, int py, int pz, const std::vector<double> &X,
                                                    const std::vector<double> &Y, const std::vector<double> &Z,
                                                    const std::vector<double> &stencil,
                                                    const std::vector<uint8_t> &dirichlet) {
  struct Entry {
    int px, py, pz;
    std::vector<double> X, Y, Z, stencil;
    std::vector<uint8_t> dirichlet;
    std::shared_ptr<const MgHierarchy> h;
  };
  static std::mutex mutex;
  static std::list<Entry> cache;  // most recent first
  constexpr size_t kEntries = 4;
  {
    std::lock_guard<std::mutex> lock(mutex);
    for (auto it = cache.begin(); it != cache.end(); ++it)
      if (it->px == px && it->py == py && it->pz == pz && it->X == X && it->Y == Y && it->Z == Z &&
          it->dirichlet == dirichlet && it->stencil == stencil) {
        cache.splice(cache.begin(), cache, it);
        return cache.front().h;
      }
  }
  std::shared_ptr<const MgHierarchy> h;
  try {
    h = std::make_shared<const MgHierarchy>(MgHierarchy::build(px, py, pz, X, Y, Z, stencil, dirichlet));
  } catch (const std::logic_error &) {
    return nullptr;
  } catch (const std::runtime_error &) {
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(mutex);
  cache.push_front(Entry{px, py, pz, X, Y, Z, stencil, dirichlet, h});
  if (cache.size() > kEntries) cache.pop_back();
  return h;
}

void free_mesh(mcb200_ctx *c) {
  for (void *p : c->mesh_owned) cudaFree(p);
  c->mesh_owned.clear();
  c->mr = MrScratch{};
}

// The refresh targets stay on the device and are uploaded when they change,
// on the upload stream: a copy from pageable host memory returns only when
// its stream reaches it, and on the context's stream that means after every
// step queued there (in a batch, the batched steps).  The upload follows the
// last refresh that read the targets; the next refresh follows the upload.
void upload_refresh_targets(mcb200_ctx *c, const int32_t *desired_e, const int32_t *desired_h) {
  MrScratch &w = c->mr;
  const int cells = c->ncells;
  if (w.de_host.size() == (size_t)cells && std::memcmp(w.de_host.data(), desired_e, sizeof(int) * cells) == 0 &&
      std::memcmp(w.dh_host.data(), desired_h, sizeof(int) * cells) == 0)
    return;
  w.de_host.assign(desired_e, desired_e + cells);
  w.dh_host.assign(desired_h, desired_h + cells);
  ck(cudaStreamWaitEvent(c->upload, c->ev_mr_used, 0), "wait");
  ck(cudaMemcpyAsync(w.de, w.de_host.data(), sizeof(int) * cells, cudaMemcpyHostToDevice, c->upload), "copy");
  ck(cudaMemcpyAsync(w.dh, w.dh_host.data(), sizeof(int) * cells, cudaMemcpyHostToDevice, c->upload), "copy");
  ck(cudaEventRecord(c->ev_upload, c->upload), "event");
  ck(cudaStreamWaitEvent(c->stream, c->ev_upload, 0), "wait");
}

void join_stat(mcb200_ctx *c) {
  if (!c->stat_pending) return;
  ck(cudaStreamWaitEvent(c->stream, c->ev_stat, 0), "wait");
  c->stat_pending = false;
}

// MultipleRefresh scratch for the mesh's cells, allocated with the cells
// (an allocation at the first refresh would stall a running batch).
void mr_scratch(mcb200_ctx *c) {
  MrScratch &w = c->mr;
  const int cells = c->ncells;
  if (w.cells == cells) return;
  w.de = dalloc<int>(cells, c->mesh_owned);
  w.dh = dalloc<int>(cells, c->mesh_owned);
  w.out_count = dalloc<unsigned int>(cells, c->mesh_owned);
  w.new_count = dalloc<unsigned int>(cells, c->mesh_owned);
  w.out_off = dalloc<unsigned int>(cells, c->mesh_owned);
  w.uid_off = dalloc<unsigned int>(cells, c->mesh_owned);
  w.tiles = dalloc<unsigned int>((cells + 1023) / 1024 + 1, c->mesh_owned);
  w.tot = dalloc<unsigned int>(2, c->mesh_owned);
  w.gen = dalloc<unsigned long long>(1, c->mesh_owned);
  w.order = dalloc<unsigned long long>(std::max<size_t>(c->capacity, 1), c->mesh_owned);
  w.wsum = dalloc<double>(std::max<size_t>(c->capacity, 1), c->mesh_owned);
  w.widx = dalloc<int>(std::max<size_t>(c->capacity, 1), c->mesh_owned);
  w.cells = cells;
  w.de_host.clear();
  w.dh_host.clear();
}

// Host particles (absolute FP64 positions) into store 0 of precision R;
// an FP32 store keeps positions relative to the cell's low corner.
template <typename R>
void upload_store(mcb200_ctx *c, size_t n, const mcb200_particles *p, const std::vector<uint32_t> &cell,
                  const std::vector<uint32_t> &meta) {
  const DevParticlesT<R> &d = store<R>(c, 0);
  auto put = [&](void *dst, const void *src, size_t sz) {
    ck(cudaMemcpyAsync(dst, src, n * sz, cudaMemcpyHostToDevice, c->stream), "upload particles");
  };
  std::vector<float> h[6];
  if constexpr (sizeof(R) == 8) {
    put(d.x, p->x, 8); put(d.y, p->y, 8); put(d.z, p->z, 8);
    put(d.kx, p->kx, 8); put(d.ky, p->ky, 8); put(d.kz, p->kz, 8);
  } else {
    for (auto &v : h) v.resize(n);
    for (size_t q = 0; q < n; ++q) {
      h[0][q] = (float)(p->x[q] - c->hlx[p->i[q]]);
      h[1][q] = (float)(p->y[q] - c->hly[p->j[q]]);
      h[2][q] = (float)(p->z[q] - c->hlz[p->k[q]]);
      h[3][q] = (float)p->kx[q]; h[4][q] = (float)p->ky[q]; h[5][q] = (float)p->kz[q];
    }
    put(d.x, h[0].data(), 4); put(d.y, h[1].data(), 4); put(d.z, h[2].data(), 4);
    put(d.kx, h[3].data(), 4); put(d.ky, h[4].data(), 4); put(d.kz, h[5].data(), 4);
  }
  put(d.energy, p->energy, 8); put(d.charge, p->charge, 8);
  put(d.cell, cell.data(), 4); put(d.itet, p->itet, 4); put(d.meta, meta.data(), 4); put(d.uid, p->uid, 4);
  ck(cudaStreamSynchronize(c->stream), "sync");
}

// The current store back to host particles (absolute FP64 positions).
template <typename R>
void download_store(mcb200_ctx *c, size_t n, mcb200_particles *p, std::vector<uint32_t> &cell,
                    std::vector<uint32_t> &meta) {
  const DevParticlesT<R> &d = store<R>(c, c->cur);
  auto get = [&](void *dst, const void *src, size_t sz) {
    ck(cudaMemcpyAsync(dst, src, n * sz, cudaMemcpyDeviceToHost, c->stream), "download particles");
  };
  std::vector<float> h[6];
  if constexpr (sizeof(R) == 8) {
    get(p->x, d.x, 8); get(p->y, d.y, 8); get(p->z, d.z, 8);
    get(p->kx, d.kx, 8); get(p->ky, d.ky, 8); get(p->kz, d.kz, 8);
  } else {
    for (auto &v : h) v.resize(n);
    get(h[0].data(), d.x, 4); get(h[1].data(), d.y, 4); get(h[2].data(), d.z, 4);
    get(h[3].data(), d.kx, 4); get(h[4].data(), d.ky, 4); get(h[5].data(), d.kz, 4);
  }
  get(p->energy, d.energy, 8); get(p->charge, d.charge, 8);
  get(cell.data(), d.cell, 4); get(p->itet, d.itet, 4); get(meta.data(), d.meta, 4); get(p->uid, d.uid, 4);
  ck(cudaStreamSynchronize(c->stream), "sync");
  if constexpr (sizeof(R) == 4) {
    for (size_t q = 0; q < n; ++q) {
      p->x[q] = c->hlx[cell[q] & 1023] + (double)h[0][q];
      p->y[q] = c->hly[(cell[q] >> 10) & 1023] + (double)h[1][q];
      p->z[q] = c->hlz[(cell[q] >> 20) & 1023] + (double)h[2][q];
      p->kx[q] = h[3][q]; p->ky[q] = h[4][q]; p->kz[q] = h[5][q];
    }
  }
}

// Stream, particle store, copy buffers, tallies and counters of a context
// on its device (the tables are already there).
void init_device_context(mcb200_ctx *c, size_t max_particles) {
  ck(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "cudaStreamCreate");
  ck(cudaStreamCreateWithFlags(&c->upload, cudaStreamNonBlocking), "cudaStreamCreate");
  ck(cudaEventCreateWithFlags(&c->ev_upload, cudaEventDisableTiming), "cudaEventCreate");
  ck(cudaEventCreateWithFlags(&c->ev_mr_used, cudaEventDisableTiming), "cudaEventCreate");
  ck(cudaStreamCreateWithFlags(&c->aux, cudaStreamNonBlocking), "cudaStreamCreate");
  ck(cudaEventCreateWithFlags(&c->ev_aux_in, cudaEventDisableTiming), "cudaEventCreate");
  ck(cudaEventCreateWithFlags(&c->ev_stat, cudaEventDisableTiming), "cudaEventCreate");
  ck(cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, c->device), "device attribute");
  c->capacity = max_particles;
  c->child_cap = (int)std::min<size_t>(std::max<size_t>(max_particles / 8, 4096), 1u << 22);
  alloc_stores(c);
  c->append_count = dalloc<unsigned int>(1, c->owned);
  c->bounds = dalloc<unsigned long long>(4, c->owned);
  ck(cudaMemsetAsync(c->bounds, 0, 4 * sizeof(unsigned long long), c->stream), "memset");
  c->tickets = dalloc<unsigned int>(1 + mcb200_ctx::kGenerations, c->owned);
  c->y.counters = dalloc<unsigned long long>(kCntNumCounters, c->owned);
  c->y.contact = dalloc<long long>(kMaxContacts * 6, c->owned);
  c->total = dalloc<unsigned int>(1, c->owned);
  c->finish_blocks = dalloc<unsigned int>(2, c->owned);
  ck(cudaMemsetAsync(c->finish_blocks, 0, 2 * sizeof(unsigned int), c->stream), "memset");
  c->dev_counts = dalloc<unsigned int>(4, c->owned);
  c->dev_psteps = dalloc<unsigned long long>(1, c->owned);
  c->sink_count = dalloc<unsigned int>(1, c->owned);
  ck(cudaMemsetAsync(c->dev_counts, 0, 4 * sizeof(unsigned int), c->stream), "memset");
  ck(cudaMemsetAsync(c->dev_psteps, 0, sizeof(unsigned long long), c->stream), "memset");
  ck(cudaMallocHost(&c->h_pinned, 64 * sizeof(unsigned int)), "cudaMallocHost");
  ck(cudaMallocHost(&c->h_scratch, 16 * sizeof(double)), "cudaMallocHost");
  ck(cudaMemsetAsync(c->y.counters, 0, sizeof(unsigned long long) * kCntNumCounters, c->stream), "memset");
  ck(cudaMemsetAsync(c->y.contact, 0, sizeof(long long) * kMaxContacts * 6, c->stream), "memset");
  ck(cudaStreamSynchronize(c->stream), "sync");
}

template <typename R>
void step_impl(mcb200_ctx *c, uint32_t step, uint64_t seed, double dt);

}  // namespace mcb200::eng

extern "C" {

int mcb200_create(const char *table_dir, double kelvin, int device, size_t max_particles, mcb200_ctx **out) {
  if (!out || !table_dir || max_particles == 0) return MCB200_ERR_ARG;
  *out = nullptr;
  mcb200_ctx *c = new mcb200_ctx;
  c->device = device;
  c->ts = std::make_shared<TableSet>();
  try {
    c->ts->tab = FullBandTables::build(table_dir, kelvin);
  } catch (const std::exception &e) {
    c->device = -1;
    int code = fail(c, MCB200_ERR_IO, e.what());
    *out = c;
    return code;
  }
  *out = c;
  if (device < 0) return MCB200_OK;  // host-only context: tables are built, nothing is uploaded
  try {
    ck(cudaSetDevice(device), "cudaSetDevice");
    c->ts->device = device;
    upload_tables(c);
    init_device_context(c, max_particles);
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
  return MCB200_OK;
}

int mcb200_create_alike(const mcb200_ctx *like, size_t max_particles, mcb200_ctx **out) {
  if (!out || !like || max_particles == 0) return MCB200_ERR_ARG;
  *out = nullptr;
  if (like->device < 0 || !like->ts || like->ts->device < 0) return MCB200_ERR_STATE;
  mcb200_ctx *c = new mcb200_ctx;
  c->device = like->device;
  c->ts = like->ts;  // the same band tables, host and device
  *out = c;
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    init_device_context(c, max_particles);
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
  return MCB200_OK;
}

void mcb200_destroy(mcb200_ctx *ctx) { delete ctx; }

int mcb200_set_flight_precision(mcb200_ctx *c, int precision) {
  if (!c || (precision != MCB200_FLIGHT_FP64 && precision != MCB200_FLIGHT_FP32)) return MCB200_ERR_ARG;
  if (c->device < 0) return fail(c, MCB200_ERR_STATE, "host-only context");
  try {
    pull_counts(c);
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CAPACITY, e.what());
  }
  if (c->n != 0) return fail(c, MCB200_ERR_STATE, "flight precision can only change while the store is empty");
  if (precision == c->precision) return MCB200_OK;
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    ck(cudaStreamSynchronize(c->stream), "sync");
    c->precision = precision;
    c->cur = 0;
    alloc_stores(c);
    ck(cudaMemsetAsync(c->bounds, 0, 4 * sizeof(unsigned long long), c->stream), "memset");  // an empty store
    return MCB200_OK;
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_get_flight_precision(const mcb200_ctx *c) { return c ? c->precision : -1; }

int mcb200_set_sort_bucket(mcb200_ctx *c, int cells_per_bucket) {
  if (!c || cells_per_bucket < 1 || cells_per_bucket > 64 || (cells_per_bucket & (cells_per_bucket - 1)))
    return MCB200_ERR_ARG;
  int shift = 0;
  while ((1 << shift) < cells_per_bucket) ++shift;
  c->sort_shift = shift;  // read when the next step's sort is launched (or captured)
  return MCB200_OK;
}

int mcb200_get_sort_bucket(const mcb200_ctx *c) { return c ? 1 << c->sort_shift : -1; }

const char *mcb200_last_error(const mcb200_ctx *ctx) { return ctx ? ctx->error.c_str() : "null context"; }

int mcb200_units(const mcb200_ctx *c, double *out, int n) {
  if (!c || !out) return MCB200_ERR_ARG;
  const Units &u = c->ts->tab.u;
  const double v[14] = {u.T0, u.eV0, u.spr0, u.time0, u.conc0, u.field0, u.scrt0,
                        u.pot0, u.a0pi, u.sieg, u.eps_silicon, u.eps_oxide, u.curr0, u.dens0};
  for (int i = 0; i < n && i < 14; ++i) out[i] = v[i];
  return MCB200_OK;
}

int mcb200_get_mesh_dims(const mcb200_ctx *c, int *nx, int *ny, int *nz) {
  if (!c || !nx || !ny || !nz) return MCB200_ERR_ARG;
  if (!c->mesh_set) return MCB200_ERR_STATE;
  *nx = c->mesh.nx;
  *ny = c->mesh.ny;
  *nz = c->mesh.nz;
  return MCB200_OK;
}

int mcb200_copy_table(const mcb200_ctx *c, const char *name, void *out, size_t bytes, size_t *needed) {
  if (!c || !name || !needed) return MCB200_ERR_ARG;
  const FullBandTables &t = c->ts->tab;
  const std::string n(name);
  std::vector<int> iv;
  std::vector<double> dv;
  if (n == "gamtet") { copy_vec(t.gamtet, out, bytes, needed); return 0; }
  if (n == "vt") { copy_vec(t.vt, out, bytes, needed); return 0; }
  if (n == "vgt") { copy_vec(t.vgt, out, bytes, needed); return 0; }
  if (n == "datantlin") { copy_vec(t.datantlin, out, bytes, needed); return 0; }
  if (n == "faclow") { copy_vec(t.faclow, out, bytes, needed); return 0; }
  if (n == "facmedium") { copy_vec(t.facmedium, out, bytes, needed); return 0; }
  if (n == "fachigh") { copy_vec(t.fachigh, out, bytes, needed); return 0; }
  if (n == "tet") { copy_vec(t.tet, out, bytes, needed); return 0; }
  if (n == "NeibrTet") { copy_vec(t.neib, out, bytes, needed); return 0; }
  if (n == "ibt") { copy_vec(t.ibt, out, bytes, needed); return 0; }
  if (n == "xkk") { copy_vec(t.xkk, out, bytes, needed); return 0; }
  if (n == "ykk") { copy_vec(t.ykk, out, bytes, needed); return 0; }
  if (n == "zkk") { copy_vec(t.zkk, out, bytes, needed); return 0; }
  if (n == "eek") { copy_vec(t.eek, out, bytes, needed); return 0; }
  if (n == "ni") { copy_vec(std::vector<double>{t.ni}, out, bytes, needed); return 0; }
  if (n == "ntlist") { copy_vec(t.ntlist, out, bytes, needed); return 0; }
  if (n == "ptlist") { copy_vec(t.ptlist, out, bytes, needed); return 0; }
  if (n == "tlist") { copy_vec(t.tlist, out, bytes, needed); return 0; }
  if (n == "nslist") { copy_vec(t.nslist, out, bytes, needed); return 0; }
  if (n == "pslist") { copy_vec(t.pslist, out, bytes, needed); return 0; }
  if (n == "dispersion") { copy_vec(t.dispersion, out, bytes, needed); return 0; }
  if (n == "slist") { copy_vec(t.slist, out, bytes, needed); return 0; }
  if (n == "ntlists") { copy_vec(t.ntlists, out, bytes, needed); return 0; }
  if (n == "ptlists") { copy_vec(t.ptlists, out, bytes, needed); return 0; }
  if (n == "tlists") { copy_vec(t.tlists, out, bytes, needed); return 0; }
  if (n == "dos") { copy_vec(t.dos, out, bytes, needed); return 0; }
  if (n == "sumdos") { copy_vec(t.sumdos, out, bytes, needed); return 0; }
  if (n == "dostetmax") { copy_vec(t.dostetmax, out, bytes, needed); return 0; }
  if (n == "sumscatt") { copy_vec(t.sumscatt, out, bytes, needed); return 0; }
  if (n == "scatte") { copy_vec(t.scatte, out, bytes, needed); return 0; }
  if (n == "dose") { copy_vec(t.dose, out, bytes, needed); return 0; }
  if (n == "scattiie") { copy_vec(t.scattiie, out, bytes, needed); return 0; }
  if (n == "scatth") { copy_vec(t.scatth, out, bytes, needed); return 0; }
  if (n == "dosh") { copy_vec(t.dosh, out, bytes, needed); return 0; }
  if (n == "scattiih") { copy_vec(t.scattiih, out, bytes, needed); return 0; }
  if (n == "energy") { copy_vec(t.energy, out, bytes, needed); return 0; }
  if (n == "matsym") { iv.assign(&t.matsym[0][0], &t.matsym[0][0] + 6 * 48); copy_vec(iv, out, bytes, needed); return 0; }
  if (n == "indmat") { iv.assign(t.indmat, t.indmat + 729); copy_vec(iv, out, bytes, needed); return 0; }
  if (n == "newisym") { iv.assign(&t.newisym[0][0], &t.newisym[0][0] + 5 * 48); copy_vec(iv, out, bytes, needed); return 0; }
  if (n == "xbz") { dv.assign(&t.xbz[0][0], &t.xbz[0][0] + 5 * 48); copy_vec(dv, out, bytes, needed); return 0; }
  if (n == "ybz") { dv.assign(&t.ybz[0][0], &t.ybz[0][0] + 5 * 48); copy_vec(dv, out, bytes, needed); return 0; }
  if (n == "zbz") { dv.assign(&t.zbz[0][0], &t.zbz[0][0] + 5 * 48); copy_vec(dv, out, bytes, needed); return 0; }
  return fail(const_cast<mcb200_ctx *>(c), MCB200_ERR_ARG, "unknown table " + n);
}

int mcb200_set_mesh(mcb200_ctx *c, int nx, int ny, int nz, const double *lx, const double *ly, const double *lz,
                    const double *wx, const double *wy, const double *wz) {
  if (c && c->device < 0) return fail(c, MCB200_ERR_STATE, "host-only context");
  if (!c || nx <= 0 || ny <= 0 || nz <= 0 || nx > 1023 || ny > 1023 || nz > 1023 || !lx || !ly || !lz)
    return c ? fail(c, MCB200_ERR_ARG, "bad mesh") : MCB200_ERR_ARG;
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    ck(cudaStreamSynchronize(c->stream), "sync");
    free_mesh(c);
    c->hlx.assign(lx, lx + nx + 1);
    c->hly.assign(ly, ly + ny + 1);
    c->hlz.assign(lz, lz + nz + 1);
    std::vector<double> dx(nx), dy(ny), dz(nz);
    for (int i = 0; i < nx; ++i) dx[i] = wx ? wx[i] : c->hlx[i + 1] - c->hlx[i];
    for (int i = 0; i < ny; ++i) dy[i] = wy ? wy[i] : c->hly[i + 1] - c->hly[i];
    for (int i = 0; i < nz; ++i) dz[i] = wz ? wz[i] : c->hlz[i + 1] - c->hlz[i];
    c->hdx = dx;
    c->hdy = dy;
    c->hdz = dz;
    DevMesh &m = c->mesh;
    m = DevMesh{};
    m.nx = nx; m.ny = ny; m.nz = nz;
    m.lx = dupload(c->hlx, c->mesh_owned); m.ly = dupload(c->hly, c->mesh_owned); m.lz = dupload(c->hlz, c->mesh_owned);
    m.dx = dupload(dx, c->mesh_owned); m.dy = dupload(dy, c->mesh_owned); m.dz = dupload(dz, c->mesh_owned);
    m.dxf = dupload(to_float(dx), c->mesh_owned);
    m.dyf = dupload(to_float(dy), c->mesh_owned);
    m.dzf = dupload(to_float(dz), c->mesh_owned);
    const size_t cells = (size_t)nx * ny * nz, nodes = (size_t)(nx + 1) * (ny + 1) * (nz + 1);
    c->ncells = (int)cells;
    m.motion = dalloc<int>(cells * 6, c->mesh_owned);
    m.contact = dalloc<int>(cells, c->mesh_owned);
    m.in_surf = dalloc<int>(cells, c->mesh_owned);
    m.nearest_surf = dalloc<int>(cells, c->mesh_owned);
    m.efield = dalloc<double>(cells * 3, c->mesh_owned);
    m.hfield = dalloc<double>(cells * 3, c->mesh_owned);
    m.rho = dalloc<double>(cells, c->mesh_owned);
    m.da = dalloc<double>(cells, c->mesh_owned);
    m.e_rough = dalloc<double>(cells, c->mesh_owned);
    m.e_sphon = dalloc<double>(cells, c->mesh_owned);
    m.h_rough = dalloc<double>(cells, c->mesh_owned);
    m.h_sphon = dalloc<double>(cells, c->mesh_owned);
    for (const void *p : {(const void *)m.e_rough, (const void *)m.e_sphon, (const void *)m.h_rough, (const void *)m.h_sphon})
      ck(cudaMemsetAsync(const_cast<void *>(p), 0, cells * sizeof(double), c->stream), "memset");
    c->y.lcurrent = dalloc<long long>(ny + 1, c->mesh_owned);
    c->y.rcurrent = dalloc<long long>(ny + 1, c->mesh_owned);
    c->y.heat_e = dalloc<long long>(nodes, c->mesh_owned);
    c->y.heat_h = dalloc<long long>(nodes, c->mesh_owned);
    c->cell32 = dalloc<float4>(cells * 3, c->mesh_owned);
    c->sb.nodes = (int)nodes;
    c->sb.node = dalloc<long long>(nodes * 10, c->mesh_owned);
    c->sb.cell_count = dalloc<unsigned long long>(cells, c->mesh_owned);
    c->sb.pot_sum = dalloc<double>(nodes, c->mesh_owned);
    c->sb.qc_pot_sum = dalloc<double>(nodes, c->mesh_owned);
    c->induced_contact = -1;
    c->induced_field = nullptr;
    c->ib = InducedBuffers{};
    c->qc = QuantumDevice{};
    c->qc_pot = nullptr;
    c->pot_scratch = nullptr;
    c->qc_set = c->qc_on = false;
    c->stat_bounds = dalloc<unsigned long long>(4, c->mesh_owned);
    c->eeff_dev = dalloc<int>(cells, c->mesh_owned);
    c->eeff_host.clear();
    c->surf_cached = false;
    c->stat_open = false;
    m.cell32 = c->cell32;
    c->hist = dalloc<unsigned int>(cells, c->mesh_owned);
    ck(cudaMemsetAsync(c->hist, 0, sizeof(unsigned int) * cells, c->stream), "memset");  // zero between sorts
    c->offsets = dalloc<unsigned int>(cells, c->mesh_owned);
    c->tile_sums = dalloc<unsigned int>((cells + 1023) / 1024 + 1, c->mesh_owned);
    ck(cudaStreamSynchronize(c->stream), "sync");
    c->mesh_set = true;
    c->cells_set = c->fields_set = c->device_set = false;
    c->fb = FieldBuffers{};
    c->cg_plan = CgPlan{};
    c->cg_plan.method = c->cg_method;
    c->cg_plan.blocks = c->cg_blocks;
    return mcb200_reset_tallies(c);
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_set_cells(mcb200_ctx *c, const int32_t *motion_rule, const int32_t *attached_contact,
                     const int32_t *in_surf_region, const int32_t *nearest_surf, const int32_t *surface_dir,
                     int n_surface_dir, const double *da, int flags) {
  if (!c) return MCB200_ERR_ARG;
  if (!c->mesh_set) return fail(c, MCB200_ERR_STATE, "mcb200_set_cells before mcb200_set_mesh");
  if (!motion_rule || !da || n_surface_dir < 0 || n_surface_dir > kMaxSurfaces)
    return fail(c, MCB200_ERR_ARG, "mcb200_set_cells: motion_rule and da are required");
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    const size_t cells = (size_t)c->ncells;
    DevMesh &m = c->mesh;
    ck(cudaMemcpy(const_cast<int *>(m.motion), motion_rule, cells * 6 * sizeof(int), cudaMemcpyHostToDevice), "copy");
    auto put_i = [&](const int *dst, const int32_t *src) {
      if (src) ck(cudaMemcpy(const_cast<int *>(dst), src, cells * sizeof(int), cudaMemcpyHostToDevice), "copy");
      else ck(cudaMemset(const_cast<int *>(dst), 0, cells * sizeof(int)), "memset");
    };
    put_i(m.contact, attached_contact);
    put_i(m.in_surf, in_surf_region);
    put_i(m.nearest_surf, nearest_surf);
    ck(cudaMemcpy(const_cast<double *>(m.da), da, cells * sizeof(double), cudaMemcpyHostToDevice), "copy");
    for (int s = 0; s < kMaxSurfaces; ++s) m.surface_dir[s] = (surface_dir && s < n_surface_dir) ? surface_dir[s] : 0;
    m.surface_scatter = (flags & MCB200_FLAG_SURFACE_SCATTER) ? 1 : 0;
    m.surface_impurity = (flags & MCB200_FLAG_SURFACE_IMPURITY) ? 1 : 0;
    m.heat = (flags & MCB200_FLAG_HEAT) ? 1 : 0;
    m.quantum = (flags & MCB200_FLAG_QUANTUM) ? 1 : 0;
    if (m.quantum && !c->ts->dt.disp)
      return fail(c, MCB200_ERR_STATE, "quantum correction needs the phonon dispersion tables (kloem.txt, kloab.txt, "
                                       "ktoem.txt, ktoab.txt, klaem.txt, klaab.txt in the table directory)");
    mr_scratch(c);
    c->cells_set = true;
    return MCB200_OK;
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_set_fields(mcb200_ctx *c, const double *efield_xyz, const double *hfield_xyz, const double *rho) {
  if (!c || !efield_xyz || !hfield_xyz || !rho) return MCB200_ERR_ARG;
  if (!c->mesh_set) return fail(c, MCB200_ERR_STATE, "mcb200_set_fields before mcb200_set_mesh");
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    const size_t cells = (size_t)c->ncells;
    ck(cudaMemcpyAsync(const_cast<double *>(c->mesh.efield), efield_xyz, cells * 3 * sizeof(double), cudaMemcpyHostToDevice, c->stream), "copy");
    ck(cudaMemcpyAsync(const_cast<double *>(c->mesh.hfield), hfield_xyz, cells * 3 * sizeof(double), cudaMemcpyHostToDevice, c->stream), "copy");
    ck(cudaMemcpyAsync(const_cast<double *>(c->mesh.rho), rho, cells * sizeof(double), cudaMemcpyHostToDevice, c->stream), "copy");
    ck(cudaStreamSynchronize(c->stream), "sync");
    c->fields_set = true;
    return MCB200_OK;
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_set_surface_rates(mcb200_ctx *c, const double *e_rough, const double *e_phonon, const double *h_rough,
                             const double *h_phonon) {
  if (!c || !e_rough || !e_phonon || !h_rough || !h_phonon) return MCB200_ERR_ARG;
  if (!c->mesh_set) return fail(c, MCB200_ERR_STATE, "mcb200_set_surface_rates before mcb200_set_mesh");
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    const size_t b = (size_t)c->ncells * sizeof(double);
    ck(cudaMemcpy(const_cast<double *>(c->mesh.e_rough), e_rough, b, cudaMemcpyHostToDevice), "copy");
    ck(cudaMemcpy(const_cast<double *>(c->mesh.e_sphon), e_phonon, b, cudaMemcpyHostToDevice), "copy");
    ck(cudaMemcpy(const_cast<double *>(c->mesh.h_rough), h_rough, b, cudaMemcpyHostToDevice), "copy");
    ck(cudaMemcpy(const_cast<double *>(c->mesh.h_sphon), h_phonon, b, cudaMemcpyHostToDevice), "copy");
    return MCB200_OK;
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_upload_particles(mcb200_ctx *c, size_t n, const mcb200_particles *p) {
  if (!c || !p) return MCB200_ERR_ARG;
  if (n > c->capacity) return fail(c, MCB200_ERR_CAPACITY, "more particles than the context capacity");
  if (!c->mesh_set) return fail(c, MCB200_ERR_STATE, "mcb200_upload_particles before mcb200_set_mesh");
  if (c->device < 0) return fail(c, MCB200_ERR_STATE, "host-only context");
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    join_stat(c);
    std::vector<uint32_t> cell(n), meta(n);
    uint32_t maxuid = 0;
    for (size_t q = 0; q < n; ++q) {
      const int i = p->i[q], j = p->j[q], k = p->k[q];
      if (i < 0 || j < 0 || k < 0 || i >= c->mesh.nx || j >= c->mesh.ny || k >= c->mesh.nz)
        return fail(c, MCB200_ERR_ARG, "particle outside the mesh");
      if (p->isym[q] < 0 || p->isym[q] > 47 || p->itet[q] < 0 || p->itet[q] >= c->ts->tab.nt || p->type[q] < 0 ||
          p->type[q] > 1)
        return fail(c, MCB200_ERR_ARG, "particle state out of range");
      cell[q] = pack_cell(i, j, k);
      meta[q] = (uint32_t)p->isym[q] | ((uint32_t)p->type[q] << 8);
      maxuid = std::max(maxuid, p->uid[q] + 1);
    }
    c->cur = 0;
    if (c->precision == MCB200_FLIGHT_FP32) upload_store<float>(c, n, p, cell, meta);
    else upload_store<double>(c, n, p, cell, meta);
    c->n = n;
    c->next_uid = maxuid;
    c->overflow_pending = false;
    ck(cudaMemsetAsync(c->dev_counts + 2, 0, sizeof(unsigned int), c->stream), "memset");
    push_counts(c);
    store_bounds(c);
    ck(cudaStreamSynchronize(c->stream), "sync");
    return MCB200_OK;
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_download_particles(mcb200_ctx *c, mcb200_particles *p, size_t capacity, size_t *n_out) {
  if (!c || !p) return MCB200_ERR_ARG;
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    pull_counts(c);
  } catch (const CapacityError &e) {
    return fail(c, MCB200_ERR_CAPACITY, e.what());
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
  if (n_out) *n_out = c->n;
  if (capacity < c->n) return fail(c, MCB200_ERR_CAPACITY, "host buffers smaller than the particle count");
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    const size_t n = c->n;
    std::vector<uint32_t> cell(n), meta(n);
    if (c->precision == MCB200_FLIGHT_FP32) download_store<float>(c, n, p, cell, meta);
    else download_store<double>(c, n, p, cell, meta);
    for (size_t q = 0; q < n; ++q) {
      p->i[q] = cell[q] & 1023;
      p->j[q] = (cell[q] >> 10) & 1023;
      p->k[q] = (cell[q] >> 20) & 1023;
      p->isym[q] = meta[q] & 255;
      p->type[q] = (meta[q] >> 8) & 255;
    }
    return MCB200_OK;
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

size_t mcb200_num_particles(const mcb200_ctx *cc) {
  if (!cc) return 0;
  mcb200_ctx *c = const_cast<mcb200_ctx *>(cc);  // reading the device count updates the host copy
  if (c->n_stale) {
    try {
      cudaSetDevice(c->device);
      pull_counts(c);
    } catch (const CapacityError &e) {
      c->overflow_pending = true;  // reported by the next call that returns a status
      c->error = e.what();
    } catch (const std::exception &e) {
      c->error = e.what();
    }
  }
  return c->n;
}

int mcb200_copy_ensemble(mcb200_ctx *dst, mcb200_ctx *src) {
  if (!dst || !src || dst == src) return MCB200_ERR_ARG;
  if (dst->device != src->device || dst->precision != src->precision || !dst->mesh_set || !src->mesh_set ||
      dst->mesh.nx != src->mesh.nx || dst->mesh.ny != src->mesh.ny || dst->mesh.nz != src->mesh.nz)
    return fail(dst, MCB200_ERR_ARG, "mcb200_copy_ensemble: contexts differ in device, precision or mesh");
  try {
    ck(cudaSetDevice(dst->device), "cudaSetDevice");
    join_stat(dst);
    pull_counts(src);
    ck(cudaStreamSynchronize(dst->stream), "sync");
    if (src->n > dst->capacity) return fail(dst, MCB200_ERR_CAPACITY, "mcb200_copy_ensemble: too many particles");
    const size_t n = src->n;
    auto copy = [&](void *d, const void *s, size_t bytes) {
      if (bytes) ck(cudaMemcpyAsync(d, s, bytes, cudaMemcpyDeviceToDevice, dst->stream), "copy ensemble");
    };
    auto move = [&](auto tag) {
      using R = decltype(tag);
      const DevParticlesT<R> &a = store<R>(src, src->cur), &b = store<R>(dst, 0);
      copy(b.x, a.x, n * sizeof(R)); copy(b.y, a.y, n * sizeof(R)); copy(b.z, a.z, n * sizeof(R));
      copy(b.kx, a.kx, n * sizeof(R)); copy(b.ky, a.ky, n * sizeof(R)); copy(b.kz, a.kz, n * sizeof(R));
      copy(b.energy, a.energy, n * 8); copy(b.charge, a.charge, n * 8);
      copy(b.cell, a.cell, n * 4); copy(b.itet, a.itet, n * 4); copy(b.meta, a.meta, n * 4); copy(b.uid, a.uid, n * 4);
    };
    if (dst->precision == MCB200_FLIGHT_FP32) move(float{});
    else move(double{});
    if (dst->device_set && src->device_set) {
      const size_t nodes = (size_t)(dst->mesh.nx + 1) * (dst->mesh.ny + 1) * (dst->mesh.nz + 1);
      copy(dst->fb.potential, src->fb.potential, nodes * sizeof(double));
    }
    dst->cur = 0;
    dst->n = n;
    dst->next_uid = src->next_uid;
    dst->overflow_pending = false;
    ck(cudaMemsetAsync(dst->dev_counts + 2, 0, sizeof(unsigned int), dst->stream), "memset");
    push_counts(dst);
    store_bounds(dst);
    ck(cudaStreamSynchronize(dst->stream), "sync");
    return MCB200_OK;
  } catch (const CapacityError &e) {
    return fail(dst, MCB200_ERR_CAPACITY, e.what());
  } catch (const std::exception &e) {
    return fail(dst, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_particle_steps(mcb200_ctx *c, uint64_t *total) {
  if (!c || !total) return MCB200_ERR_ARG;
  if (c->device < 0) return fail(c, MCB200_ERR_STATE, "host-only context");
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    ck(cudaMemcpyAsync(c->h_scratch, c->dev_psteps, sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream),
       "copy");
    ck(cudaStreamSynchronize(c->stream), "sync");
    std::memcpy(total, c->h_scratch, sizeof(uint64_t));
    return MCB200_OK;
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_seed_particles(mcb200_ctx *c, size_t n, const int32_t *cell_of, const double *charge, int type,
                          uint64_t seed) {
  if (!c || (n > 0 && (!cell_of || !charge)) || type < 0 || type > 1) return MCB200_ERR_ARG;
  if (!c->mesh_set || !c->cells_set) return fail(c, MCB200_ERR_STATE, "mcb200_seed_particles needs mesh and cells");
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    join_stat(c);
    pull_counts(c);
  } catch (const CapacityError &e) {
    return fail(c, MCB200_ERR_CAPACITY, e.what());
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
  if (c->n + n > c->capacity) return fail(c, MCB200_ERR_CAPACITY, "more particles than the context capacity");
  for (size_t q = 0; q < n; ++q)
    if (cell_of[q] < 0 || cell_of[q] >= c->ncells) return fail(c, MCB200_ERR_ARG, "cell index outside the mesh");
  if (n == 0) return MCB200_OK;
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    std::vector<void *> tmp;
    int *dcell = dalloc<int>(n, tmp);
    double *dq = dalloc<double>(n, tmp);
    ck(cudaMemcpyAsync(dcell, cell_of, n * sizeof(int), cudaMemcpyHostToDevice, c->stream), "copy");
    ck(cudaMemcpyAsync(dq, charge, n * sizeof(double), cudaMemcpyHostToDevice, c->stream), "copy");
    FlightCtx F;
    F.T = c->ts->dt;
    F.M = c->mesh;
    F.Y = c->y;
    F.C = DevChildren{};
    F.dt = 0;
    F.seed = seed;
    F.step = kSeedStreamStep;
    if (c->precision == MCB200_FLIGHT_FP32)
      launch_seed(F, store<float>(c, c->cur), (int)c->n, (int)n, dcell, dq, type, c->next_uid, grid_for(c, n, 256),
                  c->stream);
    else
      launch_seed(F, store<double>(c, c->cur), (int)c->n, (int)n, dcell, dq, type, c->next_uid, grid_for(c, n, 256),
                  c->stream);
    ck(cudaGetLastError(), "seed kernel");
    c->n += n;
    c->next_uid += (uint32_t)n;
    push_counts(c);
    store_bounds(c);
    ck(cudaStreamSynchronize(c->stream), "sync");
    for (void *p : tmp) cudaFree(p);
    return MCB200_OK;
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_step(mcb200_ctx *c, uint32_t step, uint64_t seed, double dt) {
  if (!c) return MCB200_ERR_ARG;
  if (!c->mesh_set || !c->cells_set || !c->fields_set)
    return fail(c, MCB200_ERR_STATE, "mcb200_step needs mesh, cells and fields");
  if (c->overflow_pending) {
    c->overflow_pending = false;
    return fail(c, MCB200_ERR_CAPACITY, "particle store full: GENERATE copies beyond the context capacity were dropped");
  }
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    if (c->precision == MCB200_FLIGHT_FP32) step_impl<float>(c, step, seed, dt);
    else step_impl<double>(c, step, seed, dt);
    return MCB200_OK;
  } catch (const CapacityError &e) {
    return fail(c, MCB200_ERR_CAPACITY, e.what());
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_set_timing(mcb200_ctx *c, int enable) {
  if (!c || enable < 0) return MCB200_ERR_ARG;
  if (c->device < 0) return fail(c, MCB200_ERR_STATE, "host-only context");
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    for (auto &q : c->ev)
      for (cudaEvent_t &e : q)
        if (!e) ck(cudaEventCreate(&e), "cudaEventCreate");
    harvest_all_timing(c);
    c->timing = enable != 0;
    c->timing_period = enable > 1 ? enable : 1;
    c->timing_count = 0;
    c->flight_ms = c->step_ms = 0;
    c->flight_launches = c->steps = c->particles_flown = c->launches = 0;
    ck(cudaMemcpyAsync(c->h_scratch, c->dev_psteps, sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream),
       "copy");
    ck(cudaStreamSynchronize(c->stream), "sync");
    std::memcpy(&c->psteps_at_timing, c->h_scratch, sizeof(unsigned long long));
    return MCB200_OK;
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_flush_l2(mcb200_ctx *c, size_t bytes) {
  if (!c || bytes == 0) return MCB200_ERR_ARG;
  if (c->device < 0) return fail(c, MCB200_ERR_STATE, "host-only context");
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    if (c->flush_bytes < bytes) {
      if (c->flush_buf) cudaFree(c->flush_buf);
      c->flush_buf = nullptr;
      c->flush_bytes = 0;
      ck(cudaMalloc(&c->flush_buf, bytes), "cudaMalloc");
      c->flush_bytes = bytes;
    }
    ck(cudaMemsetAsync(c->flush_buf, c->launches & 0xff, bytes, c->stream), "memset");
    return MCB200_OK;
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_mark(mcb200_ctx *c, int slot) {
  if (!c || slot < 0 || slot >= 8) return MCB200_ERR_ARG;
  if (c->device < 0) return fail(c, MCB200_ERR_STATE, "host-only context");
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    if (!c->marks[slot]) ck(cudaEventCreate(&c->marks[slot]), "cudaEventCreate");
    ck(cudaEventRecord(c->marks[slot], c->stream), "cudaEventRecord");
    return MCB200_OK;
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_elapsed_ms(mcb200_ctx *c, int from, int to, double *ms) {
  if (!c || !ms || from < 0 || from >= 8 || to < 0 || to >= 8) return MCB200_ERR_ARG;
  if (!c->marks[from] || !c->marks[to]) return fail(c, MCB200_ERR_STATE, "mark not recorded");
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    ck(cudaEventSynchronize(c->marks[to]), "cudaEventSynchronize");
    float f = 0;
    ck(cudaEventElapsedTime(&f, c->marks[from], c->marks[to]), "cudaEventElapsedTime");
    *ms = f;
    return MCB200_OK;
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_get_timing(const mcb200_ctx *cc, double *out, int n) {
  if (!cc || !out) return MCB200_ERR_ARG;
  mcb200_ctx *c = const_cast<mcb200_ctx *>(cc);  // outstanding event pairs are read back first
  if (c->device >= 0 && c->timing) {
    try {
      ck(cudaSetDevice(c->device), "cudaSetDevice");
      harvest_all_timing(c);
      ck(cudaMemcpyAsync(c->h_scratch, c->dev_psteps, sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream),
         "copy");
      ck(cudaStreamSynchronize(c->stream), "sync");
      unsigned long long now = 0;
      std::memcpy(&now, c->h_scratch, sizeof(now));
      c->particles_flown = now - c->psteps_at_timing;
    } catch (const std::exception &e) {
      return fail(c, MCB200_ERR_CUDA, e.what());
    }
  }
  const double v[6] = {c->flight_ms, (double)c->flight_launches, c->step_ms, (double)c->steps,
                       (double)c->particles_flown, (double)c->launches};
  for (int i = 0; i < n && i < 6; ++i) out[i] = v[i];
  return MCB200_OK;
}

int mcb200_sync(mcb200_ctx *c) {
  if (!c) return MCB200_ERR_ARG;
  if (c->stat_pending) {
    cudaSetDevice(c->device);
    cudaStreamWaitEvent(c->stream, c->ev_stat, 0);
    c->stat_pending = false;
  }
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return fail(c, MCB200_ERR_CUDA, cudaGetErrorString(e));
  try {
    pull_counts(c);
  } catch (const CapacityError &x) {
    return fail(c, MCB200_ERR_CAPACITY, x.what());
  } catch (const std::exception &x) {
    return fail(c, MCB200_ERR_CUDA, x.what());
  }
  return MCB200_OK;
}

int mcb200_get_tallies(mcb200_ctx *c, uint64_t *counters, double *contact, double *lcurrent, double *rcurrent,
                       double *heat_e, double *heat_h) {
  if (!c) return MCB200_ERR_ARG;
  if (!c->mesh_set) return fail(c, MCB200_ERR_STATE, "mcb200_get_tallies before mcb200_set_mesh");
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    ck(cudaStreamSynchronize(c->stream), "sync");
    pull_counts(c);
    if (counters) ck(cudaMemcpy(counters, c->y.counters, sizeof(uint64_t) * kCntNumCounters, cudaMemcpyDeviceToHost), "copy");
    if (contact) {
      std::vector<long long> v(kMaxContacts * 6);
      ck(cudaMemcpy(v.data(), c->y.contact, sizeof(long long) * v.size(), cudaMemcpyDeviceToHost), "copy");
      for (int i = 0; i < kMaxContacts; ++i) {
        contact[i * 6 + 0] = (double)v[i * 6 + 0];
        contact[i * 6 + 1] = (double)v[i * 6 + 1] / kChargeScale;
        contact[i * 6 + 2] = (double)v[i * 6 + 2] / kEnergyScale;
        contact[i * 6 + 3] = (double)v[i * 6 + 3];
        contact[i * 6 + 4] = (double)v[i * 6 + 4] / kChargeScale;
        contact[i * 6 + 5] = (double)v[i * 6 + 5] / kEnergyScale;
      }
    }
    auto get = [&](double *dst, const long long *src, size_t n, double scale) {
      if (!dst) return;
      std::vector<long long> v(n);
      ck(cudaMemcpy(v.data(), src, sizeof(long long) * n, cudaMemcpyDeviceToHost), "copy");
      for (size_t i = 0; i < n; ++i) dst[i] = (double)v[i] / scale;
    };
    const size_t nodes = (size_t)(c->mesh.nx + 1) * (c->mesh.ny + 1) * (c->mesh.nz + 1);
    get(lcurrent, c->y.lcurrent, c->mesh.ny + 1, kChargeScale);
    get(rcurrent, c->y.rcurrent, c->mesh.ny + 1, kChargeScale);
    get(heat_e, c->y.heat_e, nodes, kEnergyScale);
    get(heat_h, c->y.heat_h, nodes, kEnergyScale);
    return MCB200_OK;
  } catch (const CapacityError &e) {
    return fail(c, MCB200_ERR_CAPACITY, e.what());
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_tallies_enqueue(mcb200_ctx *c, int slot) {
  if (!c || slot < 0 || slot >= mcb200_ctx::kTallyRing) return MCB200_ERR_ARG;
  if (!c->mesh_set) return fail(c, MCB200_ERR_STATE, "mcb200_tallies_enqueue before mcb200_set_mesh");
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    constexpr int kRow = kMaxContacts * 6 + 1;
    if (!c->h_tally) {
      ck(cudaMallocHost(&c->h_tally, sizeof(long long) * kRow * mcb200_ctx::kTallyRing), "cudaMallocHost");
      for (cudaEvent_t &e : c->ev_tally) ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
    }
    // a slot enqueued before and not collected: its copy lands first
    if (c->tally_pending[slot]) ck(cudaEventSynchronize(c->ev_tally[slot]), "sync");
    long long *row = c->h_tally + (size_t)slot * kRow;
    ck(cudaMemcpyAsync(row, c->y.contact, sizeof(long long) * kMaxContacts * 6, cudaMemcpyDeviceToHost, c->stream),
       "copy");
    row[kMaxContacts * 6] = 0;
    // the store-full flag (dev_counts[2]) beside them
    ck(cudaMemcpyAsync(row + kMaxContacts * 6, c->dev_counts + 2, sizeof(unsigned int), cudaMemcpyDeviceToHost,
                       c->stream),
       "copy");
    ck(cudaEventRecord(c->ev_tally[slot], c->stream), "event");
    c->tally_pending[slot] = true;
    return MCB200_OK;
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_tallies_collect(mcb200_ctx *c, int slot, double *contact) {
  if (!c || slot < 0 || slot >= mcb200_ctx::kTallyRing || !contact) return MCB200_ERR_ARG;
  if (!c->tally_pending[slot]) return fail(c, MCB200_ERR_STATE, "mcb200_tallies_collect: nothing enqueued in the slot");
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    ck(cudaEventSynchronize(c->ev_tally[slot]), "sync");
    c->tally_pending[slot] = false;
    const long long *v = c->h_tally + (size_t)slot * (kMaxContacts * 6 + 1);
    for (int i = 0; i < kMaxContacts; ++i) {
      contact[i * 6 + 0] = (double)v[i * 6 + 0];
      contact[i * 6 + 1] = (double)v[i * 6 + 1] / kChargeScale;
      contact[i * 6 + 2] = (double)v[i * 6 + 2] / kEnergyScale;
      contact[i * 6 + 3] = (double)v[i * 6 + 3];
      contact[i * 6 + 4] = (double)v[i * 6 + 4] / kChargeScale;
      contact[i * 6 + 5] = (double)v[i * 6 + 5] / kEnergyScale;
    }
    if ((unsigned int)v[kMaxContacts * 6])
      return fail(c, MCB200_ERR_CAPACITY, "particle store full: GENERATE copies beyond the context capacity were dropped");
    return MCB200_OK;
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_reset_tallies(mcb200_ctx *c) {
  if (!c) return MCB200_ERR_ARG;
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    cudaStream_t s = c->stream;
    ck(cudaMemsetAsync(c->y.counters, 0, sizeof(unsigned long long) * kCntNumCounters, s), "memset");
    ck(cudaMemsetAsync(c->y.contact, 0, sizeof(long long) * kMaxContacts * 6, s), "memset");
    if (c->mesh_set) {
      const size_t nodes = (size_t)(c->mesh.nx + 1) * (c->mesh.ny + 1) * (c->mesh.nz + 1);
      ck(cudaMemsetAsync(c->y.lcurrent, 0, sizeof(long long) * (c->mesh.ny + 1), s), "memset");
      ck(cudaMemsetAsync(c->y.rcurrent, 0, sizeof(long long) * (c->mesh.ny + 1), s), "memset");
      ck(cudaMemsetAsync(c->y.heat_e, 0, sizeof(long long) * nodes, s), "memset");
      ck(cudaMemsetAsync(c->y.heat_h, 0, sizeof(long long) * nodes, s), "memset");
    }
    if (c->ib.sum) ck(cudaMemsetAsync(c->ib.sum, 0, 2 * sizeof(double), s), "memset");
    ck(cudaStreamSynchronize(s), "sync");
    return MCB200_OK;
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_set_device(mcb200_ctx *c, const int32_t *material, const double *donor, const double *acceptor,
                      int n_contacts, const double *vapp, const double *phims, int n_planes, const int32_t *planes) {
  if (!c || !material || !donor || !acceptor || n_contacts < 0 || n_contacts > kMaxContacts || n_planes < 0 ||
      (n_planes > 0 && !planes) || (n_contacts > 0 && (!vapp || !phims)))
    return c ? fail(c, MCB200_ERR_ARG, "mcb200_set_device: bad arguments") : MCB200_ERR_ARG;
  if (!c->mesh_set) return fail(c, MCB200_ERR_STATE, "mcb200_set_device before mcb200_set_mesh");
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    const DevMesh &m = c->mesh;
    std::vector<double> dx(m.nx), dy(m.ny), dz(m.nz);
    ck(cudaMemcpy(dx.data(), m.dx, dx.size() * 8, cudaMemcpyDeviceToHost), "copy");
    ck(cudaMemcpy(dy.data(), m.dy, dy.size() * 8, cudaMemcpyDeviceToHost), "copy");
    ck(cudaMemcpy(dz.data(), m.dz, dz.size() * 8, cudaMemcpyDeviceToHost), "copy");
    std::vector<ContactPlane> pl(n_planes);
    for (int q = 0; q < n_planes; ++q) {
      const int32_t *r = planes + 7 * q;
      pl[q] = ContactPlane{r[0], r[1], r[2], r[3], r[4], r[5], r[6]};
    }
    const Units &u = c->ts->tab.u;
    const double eps[6] = {0.0, u.eps_vacuum, u.eps_oxide, u.eps_silicon, 0.0, 0.0};
    const PoissonSetup s = PoissonSetup::build(m.nx, m.ny, m.nz, dx.data(), dy.data(), dz.data(), material, donor,
                                               acceptor, c->ts->tab.ni, eps, pl,
                                               std::vector<double>(vapp, vapp + n_contacts),
                                               std::vector<double>(phims, phims + n_contacts));
    const size_t cells = (size_t)c->ncells, nodes = (size_t)s.nodes();
    std::vector<double> dinv(nodes);
    for (size_t p = 0; p < nodes; ++p) dinv[p] = 1.0 / s.stencil[p * 7 + 6];
    FieldBuffers &f = c->fb;
    f.cvol = dupload(s.cvol, c->mesh_owned);
    f.pvol = dupload(s.pvol, c->mesh_owned);
    f.pdop = dupload(s.pdop, c->mesh_owned);
    f.vadd = dupload(s.vadd, c->mesh_owned);
    f.stencil = dupload(s.stencil, c->mesh_owned);
    f.diag_inv = dupload(dinv, c->mesh_owned);
    f.dirichlet = dupload(s.dirichlet, c->mesh_owned);
    f.bc_vapp = dupload(s.bc_vapp, c->mesh_owned);
    f.bc_phims = dupload(s.bc_phims, c->mesh_owned);
    f.acc_cell = dalloc<long long>(3 * cells, c->mesh_owned);
    f.acc_node = dalloc<long long>(nodes, c->mesh_owned);
    f.cell_e = dalloc<double>(cells, c->mesh_owned);
    f.cell_h = dalloc<double>(cells, c->mesh_owned);
    f.density = dalloc<double>(nodes, c->mesh_owned);
    f.rhs = dalloc<double>(nodes, c->mesh_owned);
    f.potential = dalloc<double>(nodes, c->mesh_owned);
    f.cg_r = dalloc<double>(nodes, c->mesh_owned);
    f.cg_z = dalloc<double>(nodes, c->mesh_owned);
    f.cg_p = dalloc<double>(nodes, c->mesh_owned);
    f.cg_p1 = dalloc<double>(nodes, c->mesh_owned);
    f.cg_r1 = dalloc<double>(nodes, c->mesh_owned);
    f.cg_q = dalloc<double>(nodes, c->mesh_owned);
    f.cg_part = dalloc<double>(3 * kCgMaxGrid, c->mesh_owned);  // the persistent CG's partial sums
    f.cg_scalars = dalloc<double>(16, c->mesh_owned);  // the CG scalars sc[0..9]
    f.abs_sum = c->bounds;
    // the cell and node pass clears the sums it reads: they start from zero
    ck(cudaMemset(f.acc_cell, 0, 3 * cells * sizeof(long long)), "memset");
    ck(cudaMemset(f.acc_node, 0, nodes * sizeof(long long)), "memset");
    f.poisson_stats = dalloc<double>(3, c->mesh_owned);
    ck(cudaMemset(f.poisson_stats, 0, 3 * sizeof(double)), "memset");
    ck(cudaMemset(f.potential, 0, nodes * sizeof(double)), "memset");
    ck(cudaMemset(f.density, 0, nodes * sizeof(double)), "memset");
    {  // multigrid hierarchy of the stencil, node coordinates from the cell widths
      std::vector<double> X(m.nx + 1, 0.0), Y(m.ny + 1, 0.0), Z(m.nz + 1, 0.0);
      for (int i = 0; i < m.nx; ++i) X[i + 1] = X[i] + dx[i];
      for (int j = 0; j < m.ny; ++j) Y[j + 1] = Y[j] + dy[j];
      for (int k = 0; k < m.nz; ++k) Z[k + 1] = Z[k] + dz[k];
      const std::shared_ptr<const MgHierarchy> h =
          cached_hierarchy(m.nx + 1, m.ny + 1, m.nz + 1, X, Y, Z, s.stencil, s.dirichlet);
      if (h) {  // (none: a mesh that does not coarsen, Jacobi preconditioning)
        c->mg = mg_upload(*h, s.stencil, c->mesh_owned);
        f.mg = &c->mg;
      }
    }
    c->cg_plan = CgPlan{};
    c->cg_plan.method = c->cg_method;
    c->cg_plan.blocks = c->cg_blocks;
    c->node_contact = s.contact_of;
    c->induced_contact = -1;  // a weighting field belongs to the device it was solved for
    c->device_set = true;
    return MCB200_OK;
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_ARG, e.what());
  }
}

int mcb200_deposit(mcb200_ctx *c) {
  if (!c) return MCB200_ERR_ARG;
  if (!c->device_set || !c->cells_set) return fail(c, MCB200_ERR_STATE, "mcb200_deposit needs set_device and set_cells");
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    deposit_enqueue(c, c->stream);
    return MCB200_OK;
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

// Cooperative launches of different contexts run one after another on the
// device (two partly resident cooperative grids could wait on each other):
// each solve waits for the device's last one and becomes the last one.  The
// chain is per device and process; hold the lock while enqueueing.
static std::mutex coop_chain_mutex;
static cudaEvent_t &coop_chain_event(int device) {
  static cudaEvent_t chain[64] = {};
  cudaEvent_t &last = chain[device & 63];
  if (!last) ck(cudaEventCreateWithFlags(&last, cudaEventDisableTiming), "cudaEventCreate");
  return last;
}

int mcb200_solve_poisson(mcb200_ctx *c, double rel_tol, int max_iter, int *iterations, double *rel_residual) {
  if (!c || rel_tol <= 0 || max_iter < 0) return MCB200_ERR_ARG;
  if (!c->device_set) return fail(c, MCB200_ERR_STATE, "mcb200_solve_poisson needs mcb200_set_device");
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    std::lock_guard<std::mutex> lock(coop_chain_mutex);
    cudaEvent_t &last = coop_chain_event(c->device);
    ck(cudaStreamWaitEvent(c->stream, last, 0), "wait");
    poisson_enqueue(c, c->stream, rel_tol, max_iter, iterations, rel_residual);
    ck(cudaEventRecord(last, c->stream), "event");
    return MCB200_OK;
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_set_induced_current(mcb200_ctx *c, int contact) {
  if (!c) return MCB200_ERR_ARG;
  if (!c->device_set) return fail(c, MCB200_ERR_STATE, "mcb200_set_induced_current needs mcb200_set_device");
  if (contact < 0) {
    c->induced_contact = -1;
    return MCB200_OK;
  }
  const size_t nodes = c->node_contact.size(), cells = (size_t)c->ncells;
  if (std::find(c->node_contact.begin(), c->node_contact.end(), (int8_t)contact) == c->node_contact.end())
    return fail(c, MCB200_ERR_ARG, "mcb200_set_induced_current: no node of that contact");
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    cudaStream_t s = c->stream;
    // Laplace's equation on the device's stencil: 1 on the contact's nodes,
    // 0 on every other contact, no charge, no doping, no built-in potential
    std::vector<double> bc(nodes, 0.0);
    for (size_t p = 0; p < nodes; ++p) bc[p] = c->node_contact[p] == contact ? 1.0 : 0.0;
    std::vector<void *> tmp;
    struct Free {
      std::vector<void *> &v;
      ~Free() { for (void *p : v) cudaFree(p); }
    } release{tmp};
    FieldBuffers w = c->fb;
    double *zero = dalloc<double>(nodes, tmp);
    ck(cudaMemsetAsync(zero, 0, nodes * sizeof(double), s), "memset");
    w.bc_vapp = dupload(bc, tmp);
    w.bc_phims = w.vadd = w.pdop = w.density = zero;
    w.potential = dalloc<double>(nodes, tmp);
    ck(cudaMemsetAsync(w.potential, 0, nodes * sizeof(double), s), "memset");
    w.rhs = dalloc<double>(nodes, tmp);
    w.poisson_stats = dalloc<double>(3, tmp);
    ck(cudaMemsetAsync(w.poisson_stats, 0, 3 * sizeof(double), s), "memset");
    CgPlan plan = c->cg_plan;
    launch_rhs((int)nodes, w, s);
    int its = 0;
    double res = 0;
    {
      std::lock_guard<std::mutex> lock(coop_chain_mutex);
      cudaEvent_t &last = coop_chain_event(c->device);
      ck(cudaStreamWaitEvent(s, last, 0), "wait");
      if (cg_prepare(c->mesh, w, 1e-12, s, plan) || cg_launch(c->mesh, w, 50000, s, plan))
        throw CudaError("weighting-potential solve failed");
      ck(cudaEventRecord(last, s), "event");
    }
    if (cg_finish(c->mesh, w, plan, s, c->h_scratch, &its, &res)) throw CudaError("weighting-potential solve failed");
    if (!(res <= 1e-10)) return fail(c, MCB200_ERR_STATE, "weighting-potential solve did not converge");
    if (!c->induced_field) c->induced_field = dalloc<double>(cells * 3, c->mesh_owned);
    DevMesh m = c->mesh;
    m.hfield = c->induced_field;            // E_w = -grad phi_w (the hole-felt sign)
    m.efield = dalloc<double>(cells * 3, tmp);
    launch_pot2field(m, w.potential, s);
    ck(cudaGetLastError(), "weighting field");
    std::vector<double> h(cells * 3);
    ck(cudaMemcpyAsync(h.data(), c->induced_field, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s), "copy");
    ck(cudaStreamSynchronize(s), "sync");
    double emax = 0;
    for (double v : h) emax = std::max(emax, std::fabs(v));
    if (!c->ib.sum) {
      c->ib.bounds = c->bounds;
      c->ib.acc = dalloc<long long>(1, c->mesh_owned);
      c->ib.sum = dalloc<double>(2, c->mesh_owned);
      ck(cudaMemsetAsync(c->ib.acc, 0, sizeof(long long), s), "memset");
    }
    ck(cudaMemsetAsync(c->ib.sum, 0, 2 * sizeof(double), s), "memset");
    c->ib.field = c->induced_field;
    c->ib.vmax = std::max(c->ts->vmax, 1e-300);
    c->ib.emax = std::max(emax, 1e-300);
    c->induced_contact = contact;
    return MCB200_OK;
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_get_induced_current(mcb200_ctx *c, double *sum, double *steps) {
  if (!c || !sum) return MCB200_ERR_ARG;
  if (c->induced_contact < 0) return fail(c, MCB200_ERR_STATE, "no weighting field (mcb200_set_induced_current)");
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    ck(cudaMemcpyAsync(c->h_scratch + 13, c->ib.sum, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "copy");
    ck(cudaStreamSynchronize(c->stream), "sync");
    *sum = c->h_scratch[13];
    if (steps) *steps = c->h_scratch[14];
    return MCB200_OK;
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_poisson_stats(mcb200_ctx *c, int64_t *solves, int64_t *iterations, double *max_rel_residual, int reset) {
  if (!c) return MCB200_ERR_ARG;
  if (!c->device_set) return fail(c, MCB200_ERR_STATE, "mcb200_poisson_stats needs mcb200_set_device");
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    ck(cudaMemcpyAsync(c->h_scratch + 10, c->fb.poisson_stats, 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream),
       "copy");
    ck(cudaStreamSynchronize(c->stream), "sync");
    if (solves) *solves = (int64_t)c->h_scratch[10];
    if (iterations) *iterations = (int64_t)c->h_scratch[11];
    if (max_rel_residual) *max_rel_residual = c->h_scratch[12];
    if (reset) ck(cudaMemsetAsync(c->fb.poisson_stats, 0, 3 * sizeof(double), c->stream), "memset");
    return MCB200_OK;
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_set_poisson_solver(mcb200_ctx *c, int method, int blocks) {
  if (!c || method < MCB200_POISSON_AUTO || method > MCB200_POISSON_MULTIGRID || blocks < 0 || blocks > kCgMaxGrid)
    return c ? fail(c, MCB200_ERR_ARG, "mcb200_set_poisson_solver: bad arguments") : MCB200_ERR_ARG;
  if (method == MCB200_POISSON_MULTIGRID && c->device_set && !c->fb.mg)
    return fail(c, MCB200_ERR_STATE, "mcb200_set_poisson_solver: no multigrid hierarchy for this device");
  c->cg_method = method;
  c->cg_blocks = blocks;
  c->cg_plan.method = method;
  c->cg_plan.blocks = blocks;
  c->cg_plan.grid = 0;  // re-planned by the next solve
  return MCB200_OK;
}

int mcb200_get_poisson_solver(mcb200_ctx *c, int *method_used, int *blocks, int *levels) {
  if (!c) return MCB200_ERR_ARG;
  if (method_used) *method_used = c->cg_plan.used;
  if (blocks) *blocks = c->cg_plan.grid;
  if (levels) *levels = c->fb.mg ? c->mg.levels : 0;
  return MCB200_OK;
}

int mcb200_surface_rates(mcb200_ctx *c, const mcb200_surface_params *p, const int32_t *eeff_direction) {
  if (!c || !p || !eeff_direction) return MCB200_ERR_ARG;
  if (!c->mesh_set) return fail(c, MCB200_ERR_STATE, "mcb200_surface_rates before mcb200_set_mesh");
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    const Units &u = c->ts->tab.u;
    SurfaceRateParams q{};
    q.delta = p->delta; q.ail = p->ail; q.xiph = p->xiph; q.theta = p->theta; q.gama = p->gama;
    q.nbmod = p->nbmod; q.npf = p->npf; q.pft = p->pft; q.pfn = p->pfn; q.kpha = p->kpha;
    q.roughness = p->roughness; q.phonon = p->phonon;
    q.eps_si = u.eps_silicon; q.eps_ox = u.eps_oxide; q.Tn = u.Tn; q.T0 = u.T0; q.boltz = 8.617343e-5;
    q.field0 = u.field0; q.em0 = u.em0; q.ec0 = u.ec0; q.hq0 = u.hq0; q.conc0 = u.conc0; q.sirho = u.sirho;
    q.scrt0 = u.scrt0;
    q.tn_nbmod = std::pow(q.Tn, q.nbmod);
    q.tn_224 = std::pow(q.Tn, 2.24);
    for (int t = 0; t < 2; ++t) {
      const double effmass = t == 0 ? 0.286 : 0.8;
      q.wq_c[t] = std::pow(12.0 * effmass * q.em0 * q.field0 / q.ec0 / q.hq0 / q.hq0, -1.0 / 3.0);
    }
    // the direction array stays on the device; it is uploaded when it changes
    if (c->eeff_host.size() != (size_t)c->ncells ||
        std::memcmp(c->eeff_host.data(), eeff_direction, sizeof(int) * c->ncells) != 0) {
      c->eeff_host.assign(eeff_direction, eeff_direction + c->ncells);
      ck(cudaMemcpyAsync(c->eeff_dev, c->eeff_host.data(), sizeof(int) * c->ncells, cudaMemcpyHostToDevice, c->stream),
         "copy");
    }
    c->surf_q = q;
    c->surf_cached = true;
    surface_rates_enqueue(c, c->stream);
    return MCB200_OK;
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_multiple_refresh(mcb200_ctx *c, const int32_t *desired_e, const int32_t *desired_h, uint32_t step,
                            uint64_t seed, int64_t *generated) {
  if (!c || !desired_e || !desired_h) return MCB200_ERR_ARG;
  if (!c->mesh_set) return fail(c, MCB200_ERR_STATE, "mcb200_multiple_refresh before mcb200_set_mesh");
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    join_stat(c);
    cudaStream_t s = c->stream;
    const int cells = c->ncells;
    size_t want = 0;
    for (int q = 0; q < cells; ++q) want += (size_t)std::max(desired_e[q], 0) + (size_t)std::max(desired_h[q], 0);
    if (want > c->capacity) return fail(c, MCB200_ERR_CAPACITY, "refresh targets exceed the particle capacity");
    mr_scratch(c);  // allocated with the cells (mcb200_set_cells)
    MrScratch &w = c->mr;
    int *de = w.de, *dh = w.dh;
    unsigned int *out_count = w.out_count, *new_count = w.new_count, *out_off = w.out_off, *uid_off = w.uid_off;
    unsigned int *tiles = w.tiles, *tot = w.tot;
    unsigned long long *gen = w.gen;
    upload_refresh_targets(c, desired_e, desired_h);
    ck(cudaMemsetAsync(gen, 0, sizeof(unsigned long long), s), "memset");
    // group the store by cell into the other buffer (hist = counts, offsets =
    // cell ends); the refreshed population then goes back to this buffer
    const int sorted = 1 - c->cur, other = c->cur;
    const RefreshParams r{seed, step, 2.0, 2.0, 1.0e-30};  // Rpar, Rsqr, pckill: src/mcmodel.cpp:3878-3880
    auto refresh = [&](auto tag) {
      using R = decltype(tag);
      launch_cell_sort(store<R>(c, c->cur), DevCount{c->dev_counts, nullptr, (int)c->capacity}, store<R>(c, sorted),
                       cells, c->mesh.nx, c->mesh.nz, c->hist, c->offsets, c->tile_sums, c->total, 0, nullptr,
                       grid_for(c, c->capacity, 256), s);
      const DevParticlesT<R> &P = store<R>(c, sorted);
      launch_refresh_count(P, c->offsets, c->hist, cells, de, dh, r, w.order, out_count, new_count, s);
      launch_exclusive_scan(out_count, out_off, tiles, tot, cells, s);
      launch_exclusive_scan(new_count, uid_off, tiles, tot + 1, cells, s);
      launch_refresh_emit(P, c->offsets, c->hist, cells, de, dh, r, w.order, w.wsum, w.widx, out_off, uid_off,
                          c->dev_counts + 1,
                          store<R>(c, other), gen, s);
    };
    if (c->precision == MCB200_FLIGHT_FP32) refresh(float{});
    else refresh(double{});
    ck(cudaEventRecord(c->ev_mr_used, s), "event");  // the targets are read
    ck(cudaMemsetAsync(c->hist, 0, sizeof(unsigned int) * cells, s), "memset");  // the step's sort expects zeros
    // the refreshed population's size and the uid counter, on the device
    refresh_counts_kernel<<<1, 32, 0, s>>>(c->dev_counts, tot);
    ck(cudaGetLastError(), "refresh");
    c->cur = other;
    c->n_stale = true;
    store_bounds(c);
    c->launches += 15;  // cell sort, count, two scans, emit, counts, charge bounds
    if (generated) {  // the only result that needs the host to wait
      ck(cudaMemcpyAsync(c->h_scratch + 13, gen, sizeof(long long), cudaMemcpyDeviceToHost, s), "copy");
      ck(cudaStreamSynchronize(s), "sync");
      std::memcpy(generated, c->h_scratch + 13, sizeof(long long));
    }
    return MCB200_OK;
  } catch (const CapacityError &e) {
    return fail(c, MCB200_ERR_CAPACITY, e.what());
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_set_quantum_correction(mcb200_ctx *c, const mcb200_quantum_params *p, const int32_t *material,
                                  const int32_t *quantum_region, int enable) {
  if (!c) return MCB200_ERR_ARG;
  if (c->device < 0) return fail(c, MCB200_ERR_STATE, "host-only context");
  if (!c->mesh_set) return fail(c, MCB200_ERR_STATE, "mcb200_set_quantum_correction before mcb200_set_mesh");
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    if (p) {
      if (!material || !quantum_region)
        return fail(c, MCB200_ERR_ARG, "mcb200_set_quantum_correction: material and quantum_region are required");
      QuantumParams q;
      for (int a = 0; a < 3; ++a) {
        q.ratio[a] = p->ratio[a];
        q.theta[a] = p->theta[a];
      }
      q.eb = p->eb;
      const DevMesh &m = c->mesh;
      QuantumHost h;
      try {
        h = quantum_setup(m.nx, m.ny, m.nz, c->hlx.data(), c->hly.data(), c->hlz.data(), c->hdx.data(), c->hdy.data(),
                          c->hdz.data(), material, quantum_region, q);
      } catch (const std::invalid_argument &e) {
        return fail(c, MCB200_ERR_ARG, e.what());
      }
      ck(cudaStreamSynchronize(c->stream), "sync");  // a running solve may read the previous set-up
      QuantumDevice d;
      d.px = m.nx + 1; d.py = m.ny + 1; d.pz = m.nz + 1;
      d.n_list = (int)h.list.size();
      d.list = h.list.empty() ? nullptr : dupload(h.list, c->mesh_owned);
      d.inside = dupload(h.inside, c->mesh_owned);
      d.eb = dupload(h.eb, c->mesh_owned);
      d.range = dupload(h.range, c->mesh_owned);
      d.qcl = dupload(h.qcl, c->mesh_owned);
      std::vector<int2> win(h.lower.size());
      for (size_t i = 0; i < win.size(); ++i) win[i] = make_int2(h.lower[i], h.upper[i]);
      d.window = dupload(win, c->mesh_owned);
      c->qc = d;
      if (!c->qc_pot) c->qc_pot = dalloc<double>((size_t)d.px * d.py * d.pz, c->mesh_owned);
      c->qc_set = true;
    }
    if (enable && !c->qc_set)
      return fail(c, MCB200_ERR_STATE, "mcb200_set_quantum_correction: no set-up (params, material, region)");
    const bool was = c->qc_on;
    c->qc_on = enable != 0;
    if (c->device_set && (c->qc_on != was || (p && c->qc_on))) {
      // the current potential's fields, with or without the correction, so
      // that the fields and the statistics agree before the next solve
      if (c->qc_on) {
        launch_effective_potential(c->qc, c->fb.potential, c->qc_pot, c->stream);
        launch_pot2field(c->mesh, c->fb.potential, c->stream, c->qc_pot);
      } else {
        launch_pot2field(c->mesh, c->fb.potential, c->stream);
      }
      ck(cudaGetLastError(), "quantum correction");
    }
    return MCB200_OK;
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_quantum_potential(mcb200_ctx *c, const double *potential, double *out) {
  if (!c || !potential || !out) return MCB200_ERR_ARG;
  if (!c->qc_set) return fail(c, MCB200_ERR_STATE, "mcb200_quantum_potential needs mcb200_set_quantum_correction");
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    const size_t nodes = (size_t)c->qc.px * c->qc.py * c->qc.pz;
    if (!c->pot_scratch) c->pot_scratch = dalloc<double>(2 * nodes, c->mesh_owned);
    ck(cudaMemcpyAsync(c->pot_scratch, potential, nodes * sizeof(double), cudaMemcpyHostToDevice, c->stream), "copy");
    launch_effective_potential(c->qc, c->pot_scratch, c->pot_scratch + nodes, c->stream);
    ck(cudaGetLastError(), "effective potential");
    ck(cudaMemcpyAsync(out, c->pot_scratch + nodes, nodes * sizeof(double), cudaMemcpyDeviceToHost, c->stream),
       "copy");
    ck(cudaStreamSynchronize(c->stream), "sync");
    c->launches += 2;
    return MCB200_OK;
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_set_refresh_targets(mcb200_ctx *c, const int32_t *desired_e, const int32_t *desired_h) {
  if (!c || !desired_e || !desired_h) return MCB200_ERR_ARG;
  if (!c->cells_set) return fail(c, MCB200_ERR_STATE, "mcb200_set_refresh_targets before mcb200_set_cells");
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    size_t want = 0;
    for (int q = 0; q < c->ncells; ++q)
      want += (size_t)std::max(desired_e[q], 0) + (size_t)std::max(desired_h[q], 0);
    if (want > c->capacity) return fail(c, MCB200_ERR_CAPACITY, "refresh targets exceed the particle capacity");
    mr_scratch(c);
    upload_refresh_targets(c, desired_e, desired_h);
    ck(cudaStreamSynchronize(c->upload), "sync");
    return MCB200_OK;
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_set_potential(mcb200_ctx *c, const double *potential) {
  return mcb200_set_potentials(c, potential, nullptr);
}

int mcb200_set_potentials(mcb200_ctx *c, const double *potential, const double *electron_potential) {
  if (!c || !potential) return MCB200_ERR_ARG;
  if (!c->device_set) return fail(c, MCB200_ERR_STATE, "mcb200_set_potential needs mcb200_set_device");
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    const size_t nodes = (size_t)(c->mesh.nx + 1) * (c->mesh.ny + 1) * (c->mesh.nz + 1);
    ck(cudaMemcpyAsync(c->fb.potential, potential, nodes * sizeof(double), cudaMemcpyHostToDevice, c->stream),
       "copy");
    const double *pot_e = nullptr;
    if (electron_potential) {
      if (!c->pot_scratch) c->pot_scratch = dalloc<double>(2 * nodes, c->mesh_owned);
      ck(cudaMemcpyAsync(c->pot_scratch, electron_potential, nodes * sizeof(double), cudaMemcpyHostToDevice,
                         c->stream),
         "copy");
      pot_e = c->pot_scratch;
    }
    launch_pot2field(c->mesh, c->fb.potential, c->stream, pot_e);
    ck(cudaGetLastError(), "pot2field");
    ck(cudaStreamSynchronize(c->stream), "sync");
    c->launches += 1;
    c->fields_set = true;
    return MCB200_OK;
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_set_heat_tally(mcb200_ctx *c, int enable) {
  if (!c) return MCB200_ERR_ARG;
  if (!c->cells_set) return fail(c, MCB200_ERR_STATE, "mcb200_set_heat_tally before mcb200_set_cells");
  c->mesh.heat = enable ? 1 : 0;
  return MCB200_OK;
}

int mcb200_stat_begin(mcb200_ctx *c, int window_steps) {
  if (!c || window_steps <= 0) return MCB200_ERR_ARG;
  if (!c->mesh_set) return fail(c, MCB200_ERR_STATE, "mcb200_stat_begin before mcb200_set_mesh");
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    join_stat(c);
    cudaStream_t s = c->stream;
    const int grid = grid_for(c, c->capacity, 256);
    const DevCount n{c->dev_counts, nullptr, (int)c->capacity};
    if (c->precision == MCB200_FLIGHT_FP32) launch_charge_bounds(store<float>(c, c->cur), n, c->stat_bounds, grid, s);
    else launch_charge_bounds(store<double>(c, c->cur), n, c->stat_bounds, grid, s);
    ck(cudaMemcpyAsync(c->h_scratch, c->stat_bounds, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s),
       "copy");
    ck(cudaStreamSynchronize(s), "sync");
    unsigned long long b[4];
    std::memcpy(b, c->h_scratch, sizeof(b));
    const double emax = std::max(c->ts->tab.emax, 1.0) * 2.0;
    for (int t = 0; t < 2; ++t) {
      double qmax;
      std::memcpy(&qmax, &b[t], 8);
      const double bound = std::max((double)b[2 + t] * qmax * window_steps * 4.0, 1e-300);
      auto unit = [](double bnd) { return std::ldexp(1.0, 62 - (int)std::ceil(std::log2(bnd))); };
      c->ss.q[t] = unit(bound);
      c->ss.v[t] = unit(bound * std::max(c->ts->vmax, 1e-300));
      c->ss.e[t] = unit(bound * emax);
    }
    const size_t nodes = (size_t)c->sb.nodes;
    ck(cudaMemsetAsync(c->sb.node, 0, sizeof(long long) * nodes * 10, s), "memset");
    ck(cudaMemsetAsync(c->sb.cell_count, 0, sizeof(unsigned long long) * c->ncells, s), "memset");
    ck(cudaMemsetAsync(c->sb.pot_sum, 0, sizeof(double) * nodes, s), "memset");
    ck(cudaMemsetAsync(c->sb.qc_pot_sum, 0, sizeof(double) * nodes, s), "memset");
    ck(cudaStreamSynchronize(s), "sync");
    c->stat_steps = 0;
    c->stat_open = true;
    return MCB200_OK;
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_stat_accumulate(mcb200_ctx *c) {
  if (!c) return MCB200_ERR_ARG;
  if (!c->stat_open) return fail(c, MCB200_ERR_STATE, "mcb200_stat_accumulate before mcb200_stat_begin");
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    cudaStream_t s = c->stream;
    const int grid = grid_for(c, c->capacity, 256);
    const DevCount n{c->dev_counts, nullptr, (int)c->capacity};
    // the particle sums only read the store: they run on the aux stream
    // beside the deposition / solve / surface rates that follow, and the
    // next change of the store waits for them (join_stat)
    join_stat(c);
    ck(cudaEventRecord(c->ev_aux_in, s), "event");
    ck(cudaStreamWaitEvent(c->aux, c->ev_aux_in, 0), "wait");
    if (c->precision == MCB200_FLIGHT_FP32)
      launch_statistic(store<float>(c, c->cur), n, c->mesh, c->ts->dt, c->ss, c->sb, grid, c->aux);
    else
      launch_statistic(store<double>(c, c->cur), n, c->mesh, c->ts->dt, c->ss, c->sb, grid, c->aux);
    ck(cudaEventRecord(c->ev_stat, c->aux), "event");
    c->stat_pending = true;
    if (c->device_set) {
      // statistic (src/mcmodel.cpp:1184-1199): the Poisson potential and the
      // electrons' (quantum-corrected) one
      launch_add_potential(c->sb.nodes, c->fb.potential, c->sb.pot_sum, s);
      if (c->qc_set)  // without a quantum set-up the two sums are the same
        launch_add_potential(c->sb.nodes, c->qc_on ? c->qc_pot : c->fb.potential, c->sb.qc_pot_sum, s);
    }
    ck(cudaGetLastError(), "statistic");
    c->stat_steps += 1;
    c->launches += 1 + (c->device_set ? (c->qc_set ? 2 : 1) : 0);
    return MCB200_OK;
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_stat_get(mcb200_ctx *c, const char *name, double *out, size_t n) {
  if (!c || !name || !out) return MCB200_ERR_ARG;
  if (!c->stat_open) return fail(c, MCB200_ERR_STATE, "no statistics window");
  const std::string nm(name);
  const size_t nodes = (size_t)c->sb.nodes, cells = (size_t)c->ncells;
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    join_stat(c);
    ck(cudaStreamSynchronize(c->stream), "sync");
    if (nm == "steps") {
      if (n < 1) return fail(c, MCB200_ERR_CAPACITY, "output too small");
      out[0] = c->stat_steps;
      return MCB200_OK;
    }
    if (nm == "cell_count") {
      if (n < cells) return fail(c, MCB200_ERR_CAPACITY, "output too small");
      std::vector<unsigned long long> h(cells);
      ck(cudaMemcpy(h.data(), c->sb.cell_count, cells * 8, cudaMemcpyDeviceToHost), "copy");
      for (size_t q = 0; q < cells; ++q) out[q] = (double)h[q];
      return MCB200_OK;
    }
    if (nm == "pot_sum" || nm == "qc_pot_sum") {
      if (n < nodes) return fail(c, MCB200_ERR_CAPACITY, "output too small");
      const bool qc = nm == "qc_pot_sum" && c->qc_set;
      ck(cudaMemcpy(out, qc ? c->sb.qc_pot_sum : c->sb.pot_sum, nodes * 8, cudaMemcpyDeviceToHost), "copy");
      return MCB200_OK;
    }
    // electron_* / hole_*: qvx, qvy, qvz, q, qe per node
    static const char *fields[5] = {"qvx", "qvy", "qvz", "q", "qe"};
    for (int t = 0; t < 2; ++t)
      for (int f = 0; f < 5; ++f)
        if (nm == std::string(t == 0 ? "electron_" : "hole_") + fields[f]) {
          if (n < nodes) return fail(c, MCB200_ERR_CAPACITY, "output too small");
          std::vector<long long> h(nodes);
          ck(cudaMemcpy(h.data(), c->sb.node + ((size_t)t * 5 + f) * nodes, nodes * 8, cudaMemcpyDeviceToHost),
             "copy");
          const double scale = f < 3 ? c->ss.v[t] : (f == 3 ? c->ss.q[t] : c->ss.e[t]);
          for (size_t q = 0; q < nodes; ++q) out[q] = (double)h[q] / scale;
          return MCB200_OK;
        }
    return fail(c, MCB200_ERR_ARG, "unknown statistic " + nm);
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_get_array(mcb200_ctx *c, const char *name, double *out, size_t n) {
  if (!c || !name || !out) return MCB200_ERR_ARG;
  if (!c->mesh_set) return fail(c, MCB200_ERR_STATE, "mcb200_get_array before mcb200_set_mesh");
  const std::string nm(name);
  const size_t cells = (size_t)c->ncells, nodes = (size_t)(c->mesh.nx + 1) * (c->mesh.ny + 1) * (c->mesh.nz + 1);
  const double *src = nullptr;
  size_t len = 0;
  if (nm == "rho") { src = c->mesh.rho; len = cells; }
  else if (nm == "e_rough") { src = c->mesh.e_rough; len = cells; }
  else if (nm == "e_phonon") { src = c->mesh.e_sphon; len = cells; }
  else if (nm == "h_rough") { src = c->mesh.h_rough; len = cells; }
  else if (nm == "h_phonon") { src = c->mesh.h_sphon; len = cells; }
  else if (nm == "efield") { src = c->mesh.efield; len = 3 * cells; }
  else if (nm == "hfield") { src = c->mesh.hfield; len = 3 * cells; }
  else if (c->device_set && nm == "cell_charge_e") { src = c->fb.cell_e; len = cells; }
  else if (c->device_set && nm == "cell_charge_h") { src = c->fb.cell_h; len = cells; }
  else if (c->device_set && nm == "cell_volume") { src = c->fb.cvol; len = cells; }
  else if (c->device_set && nm == "node_density") { src = c->fb.density; len = nodes; }
  else if (c->device_set && nm == "node_volume") { src = c->fb.pvol; len = nodes; }
  else if (c->device_set && nm == "node_doping") { src = c->fb.pdop; len = nodes; }
  else if (c->device_set && nm == "vadd") { src = c->fb.vadd; len = nodes; }
  else if (c->device_set && nm == "rhs") { src = c->fb.rhs; len = nodes; }
  else if (c->device_set && nm == "potential") { src = c->fb.potential; len = nodes; }
  else if (c->qc_set && nm == "qc_potential") { src = c->qc_pot; len = nodes; }
  else if (c->induced_contact >= 0 && nm == "induced_field") { src = c->induced_field; len = 3 * cells; }
  else if (c->device_set && nm == "stencil") { src = c->fb.stencil; len = 7 * nodes; }
  else return fail(c, MCB200_ERR_ARG, "unknown array " + nm);
  if (n < len) return fail(c, MCB200_ERR_CAPACITY, "output smaller than array " + nm);
  try {
    ck(cudaSetDevice(c->device), "cudaSetDevice");
    ck(cudaStreamSynchronize(c->stream), "sync");
    ck(cudaMemcpy(out, src, len * sizeof(double), cudaMemcpyDeviceToHost), "copy");
    return MCB200_OK;
  } catch (const std::exception &e) {
    return fail(c, MCB200_ERR_CUDA, e.what());
  }
}

}  // extern "C"

namespace mcb200::eng {

// One step of the store in precision R: main flight, mid-step copies
// generation by generation, uids and append, then removal of caught
// particles and the counting sort by cell.
// The Poisson solve of context c on stream s: right-hand side from the last
// deposit, CG (multigrid or Jacobi preconditioned; every iteration in one
// cooperative launch), true residual and statistics, cell fields.  With
// iterations and rel_residual null nothing waits for the GPU.  Two
// cooperative launches must not run at the same time on a device (each
// needs all its blocks resident at once, and two partly resident grids
// could wait on each other for ever): callers enqueue solves in one order.
void poisson_prepare(mcb200_ctx *c, cudaStream_t s, double rel_tol) {
  const int nodes = (c->mesh.nx + 1) * (c->mesh.ny + 1) * (c->mesh.nz + 1);
  launch_rhs(nodes, c->fb, s);
  if (cg_prepare(c->mesh, c->fb, rel_tol, s, c->cg_plan)) throw CudaError("Poisson solve failed");
}

void poisson_enqueue(mcb200_ctx *c, cudaStream_t s, double rel_tol, int max_iter, int *iterations,
                     double *rel_residual) {
  poisson_prepare(c, s, rel_tol);
  if (cg_launch(c->mesh, c->fb, max_iter, s, c->cg_plan)) throw CudaError("Poisson solve failed");
  poisson_finish(c, s, iterations, rel_residual);
}

void poisson_finish(mcb200_ctx *c, cudaStream_t s, int *iterations, double *rel_residual) {
  if (cg_finish(c->mesh, c->fb, c->cg_plan, s, c->h_scratch, iterations, rel_residual))
    throw CudaError("Poisson solve failed");
  if (c->qc_on) {  // compute_field, src/mcmodel.cpp:2240-2262
    launch_effective_potential(c->qc, c->fb.potential, c->qc_pot, s);
    launch_pot2field(c->mesh, c->fb.potential, s, c->qc_pot);
    c->launches += 2;
  } else {
    launch_pot2field(c->mesh, c->fb.potential, s);
  }
  ck(cudaGetLastError(), "pot2field");
  // rhs, the solve (Jacobi: set-up, dots, persistent CG, true residual and
  // statistics in 16 launches; multigrid: one), pot2field
  c->launches += c->cg_plan.used == kCgMultigrid ? 3 : 18;
  c->fields_set = true;
}

// Deposition of the current store (fixed-point units from its charge
// bounds, the particle pass, then cell and node sums) on stream s; nothing
// waits for the GPU.
void deposit_enqueue(mcb200_ctx *c, cudaStream_t s) {
  const int grid = grid_for(c, c->capacity, 256);
  const DevCount n{c->dev_counts, nullptr, (int)c->capacity};
  if (c->precision == MCB200_FLIGHT_FP32) launch_deposit(store<float>(c, c->cur), n, c->mesh, c->fb, grid, s);
  else launch_deposit(store<double>(c, c->cur), n, c->mesh, c->fb, grid, s);
  c->launches += 2;  // particle deposit, cell and node pass (units from the store's charge bounds)
  ck(cudaGetLastError(), "deposit");
  c->fields_set = true;
}

// Surface roughness / phonon rates with the parameters of the context's last
// mcb200_surface_rates call.
void surface_rates_enqueue(mcb200_ctx *c, cudaStream_t s) {
  const DevMesh &m = c->mesh;
  launch_surface_rates(c->ncells, c->surf_q, m.hfield, m.rho, c->eeff_dev, const_cast<double *>(m.e_rough),
                       const_cast<double *>(m.e_sphon), const_cast<double *>(m.h_rough),
                       const_cast<double *>(m.h_sphon), s);
  ck(cudaGetLastError(), "surface rates");
  c->launches += 1;
}

// Before the flights of a step: the induced-current tally (when on), work
// counters, the FP32 per-cell records, and zeroed copy counters of every
// generation and of the sink.
template <typename R>
void step_prepare(mcb200_ctx *c) {
  cudaStream_t s = c->stream;
  if (c->induced_contact >= 0) {  // the induced current of the store the step starts from
    launch_induced_current(store<R>(c, c->cur), DevCount{c->dev_counts, nullptr, (int)c->capacity}, c->mesh,
                           c->ts->dt, c->ib, grid_for(c, c->capacity, 256), s);
    c->launches += 2;
  }
  StepCounters z{c->tickets, {}, c->append_count};
  for (int g = 0; g < mcb200_ctx::kGenerations; ++g) z.count[g] = children<R>(c, g).count;
  z.count[mcb200_ctx::kGenerations] = c->sink_count;
  if constexpr (sizeof(R) == 4)  // FP32 flight reads the fields as per-cell float records
    launch_records_and_reset(c->ts->dt, c->mesh, c->cell32, c->ncells, z, s);
  else
    launch_step_reset(z, s);
  c->launches += 1;
  join_stat(c);  // the flights change the store the statistics read (the records and counters do not)
}

// After the flights of a step: uids for the surviving copies, which join the
// store; caught particles are dropped and the store is counting-sorted by
// cell; the sorted count becomes the particle count.
template <typename R>
void step_tail(mcb200_ctx *c) {
  cudaStream_t s = c->stream;
  const int cap = (int)c->capacity;
  ChildSetT<R> set;
  for (int g = 0; g < mcb200_ctx::kGenerations; ++g) set.g[g] = children<R>(c, g);
  // a step's copies are few: four blocks per SM, 32 copies a block, stride over them
  launch_append_children(set, c->dev_counts + 1, store<R>(c, c->cur), c->dev_counts, cap, c->append_count,
                         c->dev_counts + 2, 4 * c->sm_count, s);
  ck(cudaGetLastError(), "append children");
  c->launches += 1;
  const int other = 1 - c->cur;
  StepFinish fin;  // by the scatter's last block
  fin.n = c->dev_counts;
  fin.sorted_total = c->total;
  fin.next_uid = c->dev_counts + 1;
  fin.appended = c->append_count;
  fin.particle_steps = c->dev_psteps;
  fin.blocks = c->finish_blocks;
  fin.scan_blocks = c->finish_blocks + 1;
  launch_cell_sort(store<R>(c, c->cur), DevCount{c->dev_counts, c->append_count, cap}, store<R>(c, other), c->ncells,
                   c->mesh.nx, c->mesh.nz, c->hist, c->offsets, c->tile_sums, c->total, c->sort_shift, c->bounds,
                   grid_for(c, c->capacity, 256), s, fin);
  ck(cudaGetLastError(), "cell sort");
  c->launches += 3;  // histogram, scans, scatter
  c->cur = other;
  c->n_stale = true;
}

// The flights of a step on the context's stream, after step_prepare:
// 1. the main flight (copies go to generation 0); 2. the copies fly the
// rest of the step, generation by generation (a generation with no copies
// returns at once); copies of the last generation are counted in a sink,
// not flown.  ev (or null): timing events 1 and 2 around the main flight.
template <typename R>
void enqueue_flights(mcb200_ctx *c, FlightCtxT<R> F, cudaEvent_t *ev) {
  cudaStream_t s = c->stream;
  F.C = children<R>(c, 0);
  if (ev) ck(cudaEventRecord(ev[1], s), "event");
  launch_flight(F, store<R>(c, c->cur), DevCount{c->dev_counts, nullptr, (int)c->capacity}, c->tickets, c->sm_count,
                s);
  ck(cudaGetLastError(), "flight kernel");
  if (ev) ck(cudaEventRecord(ev[2], s), "event");
  c->launches += 1;
  for (int g = 0; g < mcb200_ctx::kGenerations; ++g) {
    if (g + 1 < mcb200_ctx::kGenerations) {
      F.C = children<R>(c, g + 1);
    } else {
      F.C = children<R>(c, g);
      F.C.count = c->sink_count;
      F.C.capacity = 0;
    }
    launch_child_flight(F, children<R>(c, g), c->child_cap, c->tickets + 1 + g, c->sm_count, s);
    ck(cudaGetLastError(), "child flight kernel");
    c->launches += 1;
  }
}

template <typename R>
void step_impl(mcb200_ctx *c, uint32_t step, uint64_t seed, double dt) {
  // Every size is read on the device (DevCount, child counts), so the step
  // is enqueued without waiting for the GPU.
  cudaStream_t s = c->stream;
  FlightCtxT<R> F;
  F.T = c->ts->dt;
  F.M = c->mesh;
  F.Y = c->y;
  F.dt = dt;
  F.seed = seed;
  F.step = step;
  cudaEvent_t *ev = nullptr;
  // events between kernels cost the next launch its overlap with the tail
  // of the one before: with a period, the other steps run without them
  const bool timed = c->timing && c->timing_count++ % (uint64_t)c->timing_period == 0;
  if (timed) {
    const int q = c->ev_head;
    c->ev_head = (q + 1) % mcb200_ctx::kTimingRing;
    harvest_timing(c, q);  // a slot is reused only after its step has finished
    ev = c->ev[q];
    c->ev_pending[q] = true;
    ck(cudaEventRecord(ev[0], s), "event");
  }
  step_prepare<R>(c);
  enqueue_flights<R>(c, F, ev);
  // 3.-4. append the copies, sort by cell
  step_tail<R>(c);
  if (ev) ck(cudaEventRecord(ev[3], s), "event");
  if (timed) {
    c->flight_launches += 1;
    c->steps += 1;
  }
}

template void step_prepare<float>(mcb200_ctx *);
template void step_prepare<double>(mcb200_ctx *);
template void step_tail<float>(mcb200_ctx *);
template void step_tail<double>(mcb200_ctx *);
template void enqueue_flights<float>(mcb200_ctx *, FlightCtxT<float>, cudaEvent_t *);
template void enqueue_flights<double>(mcb200_ctx *, FlightCtxT<double>, cudaEvent_t *);

}  // namespace mcb200::eng
