// engine_internal.h -- the engine context and the helpers its translation
// units share (engine.cu, batch.cu).  Not part of the C ABI.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "cell_kernels.h"
#include "engine_kernels.h"
#include "field_kernels.h"
#include "quantum_setup.h"
#include "flight_physics.cuh"
#include "fullband_tables.h"
#include "mcb200.h"
#include "mg_setup.h"
#include "poisson_setup.h"
#include "stat_kernels.h"

namespace mcb200::eng {


struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct CapacityError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

inline void ck(cudaError_t e, const char *what) {
  if (e != cudaSuccess) {
    cudaGetLastError();  // clear the latched error so the next call does not report this one
    throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
  }
}

template <typename T>
T *dalloc(size_t n, std::vector<void *> &owned) {
  void *p = nullptr;
  ck(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)), "cudaMalloc");
  owned.push_back(p);
  return static_cast<T *>(p);
}

template <typename T>
T *dupload(const std::vector<T> &v, std::vector<void *> &owned) {
  T *p = dalloc<T>(v.size(), owned);
  if (!v.empty()) ck(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), "upload table");
  return p;
}

// Arrays carved from one allocation, each on a 256-byte boundary: a store
// of a dozen arrays costs one cudaMalloc (a context's set-up otherwise
// spent tens of milliseconds in allocation calls).
class Carve {
 public:
  template <typename T>
  void add(T *&p, size_t n) {
    parts_.push_back({[&p](char *a) { p = reinterpret_cast<T *>(a); }, std::max<size_t>(n, 1) * sizeof(T)});
  }
  void commit(std::vector<void *> &owned) {
    size_t total = 0;
    for (const auto &q : parts_) total += round_up(q.bytes);
    void *base = nullptr;
    ck(cudaMalloc(&base, total), "cudaMalloc");
    owned.push_back(base);
    char *cur = static_cast<char *>(base);
    for (const auto &q : parts_) {
      q.set(cur);
      cur += round_up(q.bytes);
    }
    parts_.clear();
  }

 private:
  struct Part {
    std::function<void(char *)> set;
    size_t bytes;
  };
  static size_t round_up(size_t b) { return (b + 255) & ~size_t(255); }
  std::vector<Part> parts_;
};

template <typename R>
void alloc_particles(DevParticlesT<R> &d, size_t cap, std::vector<void *> &owned) {
  Carve k;
  k.add(d.x, cap); k.add(d.y, cap); k.add(d.z, cap);
  k.add(d.kx, cap); k.add(d.ky, cap); k.add(d.kz, cap);
  k.add(d.energy, cap); k.add(d.charge, cap);
  k.add(d.cell, cap); k.add(d.itet, cap);
  k.add(d.meta, cap); k.add(d.uid, cap);
  k.commit(owned);
}

template <typename R>
void alloc_children(DevChildrenT<R> &d, int cap, std::vector<void *> &owned) {
  Carve k;
  k.add(d.x, cap); k.add(d.y, cap); k.add(d.z, cap);
  k.add(d.kx, cap); k.add(d.ky, cap); k.add(d.kz, cap);
  k.add(d.energy, cap); k.add(d.charge, cap);
  k.add(d.left_time, cap);
  k.add(d.cell, cap); k.add(d.itet, cap);
  k.add(d.meta, cap);
  k.add(d.parent_uid, cap); k.add(d.sub, cap);
  k.add(d.count, 1);
  k.commit(owned);
  d.capacity = cap;
}

// One particle buffer / one child generation, in the context's flight
// precision (only the matching member is allocated).
struct ParticleBuffers {
  DevParticlesT<double> d{};
  DevParticlesT<float> f{};
};
struct ChildBuffers {
  DevChildrenT<double> d{};
  DevChildrenT<float> f{};
};

// MultipleRefresh scratch, sized for the mesh (mcb200_multiple_refresh).
struct MrScratch {
  int cells = 0;
  int *de = nullptr, *dh = nullptr;
  unsigned int *out_count = nullptr, *new_count = nullptr, *out_off = nullptr, *uid_off = nullptr;
  unsigned int *tiles = nullptr, *tot = nullptr;
  unsigned long long *gen = nullptr;
  unsigned long long *order = nullptr;  // [capacity]: uid << 32 | slot, each cell's particles in uid order
  double *wsum = nullptr;               // [capacity]: running sums of |q| of the particles a cell draws from
  int *widx = nullptr;                  // [capacity]: their slots
  std::vector<int> de_host, dh_host;  // the targets last uploaded to de / dh
};

// Band tables on the host and the device (mcb200_create): built once and
// shared by every context created alike (mcb200_create_alike).
struct TableSet {
  FullBandTables tab;
  DevTables dt{};
  double vmax = 0;  // largest group-velocity component of the band tables
  std::vector<void *> owned;
  int device = -1;
  ~TableSet() {
    if (device < 0) return;
    cudaSetDevice(device);
    for (void *p : owned) cudaFree(p);
  }
};

}  // namespace mcb200::eng

using namespace mcb200;
using namespace mcb200::eng;

struct mcb200_ctx {
  std::string error;
  int device = 0;
  cudaStream_t stream = nullptr;
  // uploads that must not wait for the work queued on `stream` (refresh
  // targets from pageable memory); ev_mr_used: the last refresh's reads
  cudaStream_t upload = nullptr;
  cudaEvent_t ev_upload = nullptr, ev_mr_used = nullptr;
  // the particle statistics run on `aux` beside the deposition and solve
  // (they only read the store); stat_pending until the stream has joined them
  cudaStream_t aux = nullptr;
  cudaEvent_t ev_aux_in = nullptr, ev_stat = nullptr;
  bool stat_pending = false;
  std::vector<void *> owned;   // every cudaMalloc of the context
  std::vector<void *> mesh_owned;
  std::shared_ptr<TableSet> ts;  // band tables (host and device), shared by contexts made alike
  DevMesh mesh{};
  bool mesh_set = false, cells_set = false, fields_set = false;
  std::vector<double> hlx, hly, hlz;
  std::vector<double> hdx, hdy, hdz;  // cell widths as given to mcb200_set_mesh
  // particles: two buffers, the store ping-pongs through the cell sort
  int precision = MCB200_FLIGHT_FP64;
  std::vector<void *> store_owned;  // particle and child buffers (reallocated on a precision change)
  size_t capacity = 0;
  ParticleBuffers pb[2];
  int cur = 0;
  size_t n = 0;
  uint32_t next_uid = 0;
  // mid-step copies: one buffer per generation
  static constexpr int kGenerations = kChildGenerations;
  ChildBuffers cb[kGenerations];
  int child_cap = 0;
  unsigned int *append_count = nullptr;
  // [4] charge bounds of the current store (charge_bounds_kernel's layout):
  // the step's sort computes them, every other writer of the store after it
  // writes (store_bounds); the deposition's fixed-point units come from them
  unsigned long long *bounds = nullptr;
  unsigned int *finish_blocks = nullptr;  // [2] blocks of the step's scatter / scan done (zero between steps)
  unsigned int *tickets = nullptr;  // work counters of the persistent flight launches (main + generations)
  float4 *cell32 = nullptr;         // FP32 flight's per-cell records (mesh-sized)
  // tallies
  DevTallies y{};
  // sort scratch
  unsigned int *hist = nullptr, *offsets = nullptr, *tile_sums = nullptr, *total = nullptr;
  int ncells = 0;
  unsigned int *h_pinned = nullptr;  // small pinned readback area
  MrScratch mr;                      // in mesh_owned
  // effective-potential quantum correction (mcb200_set_quantum_correction);
  // arrays in mesh_owned.  qc_on: solves give electrons the corrected field
  QuantumDevice qc;
  double *qc_pot = nullptr;
  double *pot_scratch = nullptr;  // [2][nodes]: caller potentials (mcb200_set_potentials, mcb200_quantum_potential)
  bool qc_set = false, qc_on = false;
  int sm_count = 148;
  int grid_per_sm = 8;  // blocks per SM of the grid-stride per-step kernels (sort, deposition, copies)
  int sort_shift = 0;   // the step's counting sort groups 2^sort_shift consecutive cells (mcb200_set_sort_bucket)
  // deposition / Poisson (mcb200_set_device)
  FieldBuffers fb{};
  CgPlan cg_plan;
  MgDevice mg{};                            // multigrid hierarchy of the Poisson stencil (mcb200_set_device)
  int cg_method = kCgAuto, cg_blocks = 0;   // mcb200_set_poisson_solver
  bool device_set = false;
  double *h_scratch = nullptr;  // pinned, 16 doubles
  // pipelined contact-tally readback (mcb200_tallies_enqueue / _collect):
  // kTallyRing slots of the contact tallies and the store-full flag, pinned
  static constexpr int kTallyRing = 4;
  long long *h_tally = nullptr;              // [kTallyRing][kMaxContacts * 6 + 1]
  cudaEvent_t ev_tally[kTallyRing] = {};
  bool tally_pending[kTallyRing] = {};
  // window statistics (mcb200_stat_*)
  StatBuffers sb{};
  StatScales ss{};
  unsigned long long *stat_bounds = nullptr;
  int *eeff_dev = nullptr;           // surface-normal field component per cell (mcb200_surface_rates)
  std::vector<int> eeff_host;
  bool surf_cached = false;          // surf_q holds the parameters of the last mcb200_surface_rates call
  SurfaceRateParams surf_q{};
  int stat_steps = 0;
  bool stat_open = false;
  // induced (Ramo-Shockley) current of one contact (mcb200_set_induced_current)
  std::vector<int8_t> node_contact;  // host: the contact of each Dirichlet node, -1 elsewhere
  int induced_contact = -1;
  double *induced_field = nullptr;   // [cells][3] weighting field (mesh_owned)
  InducedBuffers ib{};               // the per-step tally (bounds, fixed-point step sum, FP64 running sum)
  // device-resident counts: the step path never waits for them; `n` and
  // `next_uid` above are host copies, valid while !n_stale
  unsigned int *dev_counts = nullptr;         // [0] particles, [1] next uid, [2] store-full flag
  unsigned long long *dev_psteps = nullptr;   // particle-steps flown (particles at the start of each step)
  unsigned int *sink_count = nullptr;         // copies of the last child generation: counted, not stored
  bool n_stale = false;
  bool overflow_pending = false;              // a store-full flag seen, not yet reported
  // CUDA-event timing on the context's stream (mcb200_timing): a ring of
  // per-step event quadruples, read back when a slot is reused or on demand
  bool timing = false;
  int timing_period = 1;      // one step in timing_period is bracketed by events
  uint64_t timing_count = 0;  // steps since timing was turned on
  static constexpr int kTimingRing = 64;
  cudaEvent_t ev[kTimingRing][4] = {};
  bool ev_pending[kTimingRing] = {};
  int ev_head = 0;
  unsigned long long psteps_at_timing = 0;
  cudaEvent_t marks[8] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  void *flush_buf = nullptr;  // mcb200_flush_l2 scratch
  size_t flush_bytes = 0;
  double flight_ms = 0, step_ms = 0;
  uint64_t flight_launches = 0, steps = 0, particles_flown = 0, launches = 0;

  ~mcb200_ctx() {
    if (device < 0) return;
    cudaSetDevice(device);
    for (auto &q : ev)
      for (cudaEvent_t e : q)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : marks)
      if (e) cudaEventDestroy(e);
    for (void *p : mesh_owned) cudaFree(p);
    for (void *p : store_owned) cudaFree(p);
    for (void *p : owned) cudaFree(p);
    if (flush_buf) cudaFree(flush_buf);
    if (h_pinned) cudaFreeHost(h_pinned);
    if (h_scratch) cudaFreeHost(h_scratch);
    if (h_tally) cudaFreeHost(h_tally);
    for (cudaEvent_t e : ev_tally)
      if (e) cudaEventDestroy(e);
    if (aux) cudaStreamSynchronize(aux);
    if (ev_aux_in) cudaEventDestroy(ev_aux_in);
    if (ev_stat) cudaEventDestroy(ev_stat);
    if (aux) cudaStreamDestroy(aux);
    if (ev_upload) cudaEventDestroy(ev_upload);
    if (ev_mr_used) cudaEventDestroy(ev_mr_used);
    if (upload) cudaStreamDestroy(upload);
    if (stream) cudaStreamDestroy(stream);
  }
};

static_assert(sizeof(TetFlightT<float>) == 128, "FP32 tet record: one 128-byte line");
static_assert(sizeof(TetFlightT<double>) == 256, "FP64 tet record: two 128-byte lines");


namespace mcb200::eng {

template <typename R>
DevParticlesT<R> &store(mcb200_ctx *c, int i) {
  if constexpr (sizeof(R) == 8) return c->pb[i].d;
  else return c->pb[i].f;
}
template <typename R>
DevChildrenT<R> &children(mcb200_ctx *c, int g) {
  if constexpr (sizeof(R) == 8) return c->cb[g].d;
  else return c->cb[g].f;
}

int fail(mcb200_ctx *c, int code, const std::string &msg);
// Host copies of the device counts (waits for the stream when a step may
// have changed them); throws CapacityError once for a store-full flag.
void pull_counts(mcb200_ctx *c);
void push_counts(mcb200_ctx *c);
// The context stream waits for pending particle statistics (before anything
// that changes the particle store, resets or reads the statistics).  Never
// inside a stream capture: the batch joins its members first.
void join_stat(mcb200_ctx *c);
int grid_for(const mcb200_ctx *c, size_t n, int block);
void poisson_enqueue(mcb200_ctx *c, cudaStream_t s, double rel_tol, int max_iter, int *iterations,
                     double *rel_residual);
// poisson_enqueue around a caller's own launch of the solve: the right side
// and the CG set-up (fixes c->cg_plan), then, after the launch, the true
// residual, statistics and fields.
void poisson_prepare(mcb200_ctx *c, cudaStream_t s, double rel_tol);
void poisson_finish(mcb200_ctx *c, cudaStream_t s, int *iterations, double *rel_residual);
void surface_rates_enqueue(mcb200_ctx *c, cudaStream_t s);
void deposit_enqueue(mcb200_ctx *c, cudaStream_t s);
// The parts of a transport step around its flights (engine.cu).
template <typename R>
void step_prepare(mcb200_ctx *c);
template <typename R>
void step_tail(mcb200_ctx *c);
// The main and copy flights of a step on the context's stream (after
// step_prepare, before step_tail); ev: optional timing events.
template <typename R>
void enqueue_flights(mcb200_ctx *c, FlightCtxT<R> F, cudaEvent_t *ev);

}  // namespace mcb200::eng
