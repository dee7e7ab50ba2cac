// batch.cu -- many simulations stepped together (mcb200_batch_*).
//
// The reference runs one simulation per process.  Here independent
// simulations of uneven size (bulk boxes, FinFETs at different biases,
// different meshes and particle counts), each an mcb200_ctx made alike (the
// same band tables), take their transport step together: their flights run
// as ONE persistent launch over a per-simulation table (batch_flight_kernel,
// flight_kernels.cu), likewise each generation of copies, while the work
// before and after the flights (deposition, Poisson, fields, the counting
// sort) stays on each simulation's own stream, where simulations overlap on
// the device.  A particle's draws come from its own stream (seed, uid,
// step), so each simulation steps exactly as it would alone.
//
// Ordering: a batch step waits (on the device) for the work already enqueued
// on every member's stream, and every member's later work waits for the
// batch step, so member calls and batch steps interleave freely.
#include <map>

#include "engine_internal.h"

struct mcb200_batch {
  std::string error;
  int device = 0, precision = MCB200_FLIGHT_FP64;
  std::vector<mcb200_ctx *> m;
  std::vector<mcb200_batch_member> cfg;
  cudaStream_t stream = nullptr;
  cudaStream_t side = nullptr;  // the flight of the members not solving Poisson, beside the solves
  cudaEvent_t ev_flight = nullptr, ev_fork = nullptr, ev_solved = nullptr, ev_side = nullptr, ev_side0 = nullptr;
  std::vector<cudaEvent_t> ev_member;
  std::vector<uint32_t> member_step;  // host copy of each member's step number
  // full timesteps replayed from CUDA graphs: one per (store parity, members
  // solving Poisson), with the host-side effects of one step (launch counts)
  bool use_graphs = false;
  struct Graph {
    cudaGraphExec_t exec = nullptr;
    std::vector<uint64_t> member_launches;
    uint64_t batch_launches = 0;
  };
  std::map<std::pair<int, uint64_t>, Graph> graphs;
  uint64_t graph_replays = 0, graph_captures = 0;
  cudaEvent_t marks[8] = {};
  void *tables = nullptr;          // device: [6][n] BatchInstT (main flight x 2 parities, 4 copy generations)
  uint32_t *steps = nullptr;       // device: step number of each member
  unsigned int *tickets = nullptr;  // device: work counters of the batched launches (main, 4 copy generations, side)
  bool overlap = true;              // fly the members not solving Poisson beside the solves
  bool pair_solves = true;          // two multigrid solves of the same shape per cooperative launch
  bool smem_table = false;          // batched flights copy the member table into shared memory (else read in place)
  // members that fly in launches of their own on their own streams (bit k),
  // fixed by mcb200_batch_set_solo from the particle counts of that moment
  uint64_t solo = 0;
  size_t solo_min = 0;  // their smallest particle count (0: none solo)
  cudaEvent_t ev_steps = nullptr;  // after the step numbers advanced
  std::vector<unsigned char> snap;  // per member: DevMesh, DevTallies and store parity the tables were built for
  uint64_t steps_done = 0, built_at = 0;
  int blocks_per_sm = 0;  // batched flight grid (0: as many as fit); mcb200_batch_autotune
  uint64_t launches = 0;

  void drop_graphs() {
    for (auto &g : graphs)
      if (g.second.exec) cudaGraphExecDestroy(g.second.exec);
    graphs.clear();
  }
  ~mcb200_batch() {
    cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    drop_graphs();
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_solved) cudaEventDestroy(ev_solved);
    if (ev_side) cudaEventDestroy(ev_side);
    if (ev_side0) cudaEventDestroy(ev_side0);
    if (ev_steps) cudaEventDestroy(ev_steps);
    if (tables) cudaFree(tables);
    if (steps) cudaFree(steps);
    if (tickets) cudaFree(tickets);
    if (ev_flight) cudaEventDestroy(ev_flight);
    for (cudaEvent_t e : ev_member)
      if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : marks)
      if (e) cudaEventDestroy(e);
    if (side) cudaStreamDestroy(side);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace mcb200::eng {
namespace {

int bfail(mcb200_batch *b, int code, const std::string &msg) {
  if (b) b->error = msg;
  return code;
}

constexpr size_t kSnapBytes = sizeof(DevMesh) + sizeof(DevTallies) + sizeof(int);

void snapshot(const mcb200_ctx *c, int parity, unsigned char *out) {
  std::memcpy(out, &c->mesh, sizeof(DevMesh));
  std::memcpy(out + sizeof(DevMesh), &c->y, sizeof(DevTallies));
  std::memcpy(out + sizeof(DevMesh) + sizeof(DevTallies), &parity, sizeof(int));
}

// The six tables of the batch, for the members' current stores and meshes:
// main flight at this step's store parity and at the next, then the four
// copy generations (copies of generation g go to g + 1; the last
// generation's copies are counted in the member's sink).
template <typename R>
void build_tables(mcb200_batch *b) {
  const int n = (int)b->m.size();
  std::vector<BatchInstT<R>> t(6 * (size_t)n);
  for (int k = 0; k < n; ++k) {
    mcb200_ctx *c = b->m[k];
    BatchInstT<R> base{};
    base.M = c->mesh;
    base.Y = c->y;
    base.dt = b->cfg[k].dt;
    base.seed = b->cfg[k].seed;
    base.step = b->member_step[k];  // advanced with b->steps after every step
    base.n = c->dev_counts;
    base.capacity = (int)c->capacity;
    for (int par = 0; par < 2; ++par) {
      BatchInstT<R> e = base;
      e.P = store<R>(c, par == 0 ? c->cur : 1 - c->cur);
      e.C = children<R>(c, 0);
      t[(size_t)par * n + k] = e;
    }
    for (int g = 0; g < mcb200_ctx::kGenerations; ++g) {
      BatchInstT<R> e = base;
      e.in = children<R>(c, g);
      if (g + 1 < mcb200_ctx::kGenerations) {
        e.C = children<R>(c, g + 1);
      } else {
        e.C = children<R>(c, g);
        e.C.count = c->sink_count;
        e.C.capacity = 0;
      }
      t[(size_t)(2 + g) * n + k] = e;
    }
    snapshot(c, c->cur, &b->snap[(size_t)k * kSnapBytes]);
  }
  // the previous launches may still read the tables: replace them in order on the batch stream
  ck(cudaStreamSynchronize(b->stream), "sync");
  ck(cudaMemcpyAsync(b->tables, t.data(), t.size() * sizeof(BatchInstT<R>), cudaMemcpyHostToDevice, b->stream),
     "upload batch tables");
  ck(cudaStreamSynchronize(b->stream), "sync");
  b->built_at = b->steps_done;
  b->drop_graphs();  // they hold the old tables' layout assumptions
}

// True when every member still has the mesh, tallies and store parity the
// tables assume for this step.
bool tables_current(const mcb200_batch *b) {
  const int flip = (int)((b->steps_done - b->built_at) & 1);
  unsigned char now[kSnapBytes];
  for (size_t k = 0; k < b->m.size(); ++k) {
    const mcb200_ctx *c = b->m[k];
    const unsigned char *was = &b->snap[k * kSnapBytes];
    int built_cur = 0;
    std::memcpy(&built_cur, was + sizeof(DevMesh) + sizeof(DevTallies), sizeof(int));
    if (c->cur != (flip ? 1 - built_cur : built_cur)) return false;
    snapshot(c, built_cur, now);
    if (std::memcmp(now, was, kSnapBytes) != 0) return false;
  }
  return true;
}


void join_members(mcb200_batch *b);

uint64_t all_members(const mcb200_batch *b) {
  const size_t n = b->m.size();
  return n >= 64 ? ~0ull : (1ull << n) - 1;
}

// The transport part of a step (mcb200_step for every member): the tables
// must be current.  The members in `early` (none of them waiting for work on
// the batch stream) fly on the side stream as soon as their own streams are
// ready, one block per SM (it fits beside the 512-thread block per SM of a
// Poisson solve); the others fly in the main launch on the batch stream,
// after which a helper launch on the batch stream draws from the side
// launch's work counter with the room the solves left.  The copy
// generations of all batched members follow.  Solo members (b->solo) fly
// in launches of their own on their own streams, as mcb200_step does, with
// the step number read from b->steps.  A particle's flight does not depend
// on the launch or block that carries it.
template <typename R>
void batch_transport(mcb200_batch *b, uint64_t early = 0) {
  const int n = (int)b->m.size();
  const uint64_t all = all_members(b);
  const uint64_t solo = b->solo & all, batched = all & ~solo;
  early &= batched;
  if (early == batched) early = 0;  // one launch
  // 1. every member: counters and records for the step; a batched member's
  //    flight stream waits for it, a solo member flies on at once
  FlightCtxT<R> F;
  F.T = b->m[0]->ts->dt;
  for (int k = 0; k < n; ++k) {
    mcb200_ctx *c = b->m[k];
    step_prepare<R>(c);
    if ((solo >> k) & 1) {
      FlightCtxT<R> Fk;
      Fk.T = F.T;
      Fk.M = c->mesh;
      Fk.Y = c->y;
      Fk.dt = b->cfg[k].dt;
      Fk.seed = b->cfg[k].seed;
      Fk.step = b->member_step[k];
      Fk.step_dev = b->steps + k;  // graph replays run at later steps
      enqueue_flights<R>(c, Fk, nullptr);
      ck(cudaEventRecord(b->ev_member[k], c->stream), "event");  // its flights have read the step
      continue;
    }
    ck(cudaEventRecord(b->ev_member[k], c->stream), "event");
    ck(cudaStreamWaitEvent((early >> k) & 1 ? b->side : b->stream, b->ev_member[k], 0), "wait");
  }
  // 2. the batched flights
  const int flip = (int)((b->steps_done - b->built_at) & 1);
  const BatchInstT<R> *tab = static_cast<const BatchInstT<R> *>(b->tables);
  const int sms = b->m[0]->sm_count;
  unsigned int *side_ticket = b->tickets + 1 + mcb200_ctx::kGenerations;
  if (batched) {
    if (early) {
      ck(cudaMemsetAsync(side_ticket, 0, sizeof(unsigned int), b->side), "memset");
      ck(cudaEventRecord(b->ev_side0, b->side), "event");  // the side counter is reset
      if (launch_batch_flight<R>(F, tab + (size_t)flip * n, n, early, b->steps, false, side_ticket, 1, sms, b->side,
                                 b->smem_table))
        throw std::runtime_error("batched flight launch failed");
      ck(cudaEventRecord(b->ev_side, b->side), "event");
    }
    ck(cudaMemsetAsync(b->tickets, 0, sizeof(unsigned int) * (1 + mcb200_ctx::kGenerations), b->stream), "memset");
    if (launch_batch_flight<R>(F, tab + (size_t)flip * n, n, batched & ~early, b->steps, false, b->tickets,
                               b->blocks_per_sm, sms, b->stream, b->smem_table))
      throw std::runtime_error("batched flight launch failed");
    if (early) {  // the helper, then the side launch's end
      ck(cudaStreamWaitEvent(b->stream, b->ev_side0, 0), "wait");
      if (launch_batch_flight<R>(F, tab + (size_t)flip * n, n, early, b->steps, false, side_ticket, b->blocks_per_sm,
                                 sms, b->stream, b->smem_table))
        throw std::runtime_error("batched flight launch failed");
      ck(cudaStreamWaitEvent(b->stream, b->ev_side, 0), "wait");
    }
    for (int g = 0; g < mcb200_ctx::kGenerations; ++g)
      if (launch_batch_flight<R>(F, tab + (size_t)(2 + g) * n, n, batched, b->steps, true, b->tickets + 1 + g,
                                 b->blocks_per_sm, sms, b->stream, b->smem_table))
        throw std::runtime_error("batched copy flight launch failed");
    b->launches += 2 + mcb200_ctx::kGenerations + (early ? 2 : 0);
  }
  ck(cudaEventRecord(b->ev_flight, b->stream), "event");
  // 3. every member: its tail after its flights, on its own stream
  for (int k = 0; k < n; ++k) {
    mcb200_ctx *c = b->m[k];
    if (!((solo >> k) & 1)) ck(cudaStreamWaitEvent(c->stream, b->ev_flight, 0), "wait");
    step_tail<R>(c);
  }
  // 4. the step numbers advance once every flight has read them; the solo
  //    members' next flights wait for that
  for (int k = 0; k < n; ++k)
    if ((solo >> k) & 1) ck(cudaStreamWaitEvent(b->stream, b->ev_member[k], 0), "wait");
  launch_advance_batch_steps<R>(b->steps, static_cast<BatchInstT<R> *>(b->tables), n, 6, b->stream);
  ck(cudaGetLastError(), "advance steps");
  if (solo) {
    ck(cudaEventRecord(b->ev_steps, b->stream), "event");
    for (int k = 0; k < n; ++k)
      if ((solo >> k) & 1) ck(cudaStreamWaitEvent(b->m[k]->stream, b->ev_steps, 0), "wait");
  }
  b->steps_done += 1;
  for (uint32_t &st : b->member_step) ++st;
}

// Members that solve Poisson at this step (bit k).
uint64_t poisson_due(const mcb200_batch *b) {
  uint64_t due = 0;
  for (size_t k = 0; k < b->m.size(); ++k) {
    const mcb200_batch_member &m = b->cfg[k];
    const uint32_t every = m.poisson_every > 0 ? (uint32_t)m.poisson_every : 1u;
    if (m.self_consistent && b->m[k]->device_set && b->member_step[k] % every == 0) due |= 1ull << k;
  }
  return due;
}

// A full timestep of every member, as density() orders it: deposition,
// Poisson + fields where due (solves one after another on the batch stream:
// no two cooperative launches overlap), surface rates, then the transport
// step.  Member streams fork from the batch stream and join it at the end,
// so the step is one unit of work on the batch stream (and capturable).
template <typename R>
void batch_full_step(mcb200_batch *b, uint64_t due) {
  const int n = (int)b->m.size();
  ck(cudaEventRecord(b->ev_fork, b->stream), "event");
  for (int k = 0; k < n; ++k) {
    mcb200_ctx *c = b->m[k];
    ck(cudaStreamWaitEvent(c->stream, b->ev_fork, 0), "wait");
    if (b->cfg[k].self_consistent && c->device_set) deposit_enqueue(c, c->stream);
  }
  if (due) {
    // on the batch stream: every due member's set-up, the solves (two
    // multigrid solves of the same shape share a launch when pairing is on),
    // then the residuals and fields
    std::vector<int> solving;
    for (int k = 0; k < n; ++k) {
      if (!((due >> k) & 1)) continue;
      mcb200_ctx *c = b->m[k];
      ck(cudaEventRecord(b->ev_member[k], c->stream), "event");
      ck(cudaStreamWaitEvent(b->stream, b->ev_member[k], 0), "wait");
      poisson_prepare(c, b->stream, b->cfg[k].poisson_rel_tol > 0 ? b->cfg[k].poisson_rel_tol : 1e-10);
      solving.push_back(k);
    }
    constexpr int kMaxIter = 20000;
    std::vector<char> launched(n, 0);
    for (size_t i = 0; i < solving.size(); ++i) {
      const int k0 = solving[i];
      if (launched[k0]) continue;
      mcb200_ctx *c0 = b->m[k0];
      launched[k0] = 1;
      int k1 = -1;
      if (b->pair_solves && c0->cg_plan.used == kCgMultigrid && cg_mg_pair_fits(c0->cg_plan.grid))
        for (size_t j = i + 1; j < solving.size() && k1 < 0; ++j) {
          mcb200_ctx *c = b->m[solving[j]];
          if (!launched[solving[j]] && c->cg_plan.used == kCgMultigrid && c->cg_plan.grid == c0->cg_plan.grid &&
              c->fb.mg->levels == c0->fb.mg->levels && c->fb.mg->nu == c0->fb.mg->nu)
            k1 = solving[j];
        }
      if (k1 >= 0) {
        mcb200_ctx *c1 = b->m[k1];
        launched[k1] = 1;
        const MgSystem two[2] = {cg_mg_system(c0->mesh, c0->fb, kMaxIter, c0->cg_plan.rel_tol2),
                                 cg_mg_system(c1->mesh, c1->fb, kMaxIter, c1->cg_plan.rel_tol2)};
        ck(launch_cg_mg_pair(two, c0->cg_plan.grid, b->stream), "paired Poisson solve");
        c0->cg_plan.launches += 1;
        c1->cg_plan.launches += 1;
        b->launches += 1;
      } else if (cg_launch(c0->mesh, c0->fb, kMaxIter, b->stream, c0->cg_plan)) {
        throw CudaError("Poisson solve failed");
      }
    }
    for (int k : solving) poisson_finish(b->m[k], b->stream, nullptr, nullptr);
    ck(cudaEventRecord(b->ev_solved, b->stream), "event");
    for (int k = 0; k < n; ++k)
      if ((due >> k) & 1) ck(cudaStreamWaitEvent(b->m[k]->stream, b->ev_solved, 0), "wait");
  }
  for (int k = 0; k < n; ++k) {
    mcb200_ctx *c = b->m[k];
    if (b->cfg[k].surface_rates && c->surf_cached) surface_rates_enqueue(c, c->stream);
  }
  batch_transport<R>(b, b->overlap ? all_members(b) & ~due : 0);
  join_members(b);
}

// A graph step on the batch stream, ordered with the members' own streams:
// it follows the work already enqueued on them, and their later work (a
// refresh, a download) follows it.
void launch_graph(mcb200_batch *b, cudaGraphExec_t exec) {
  join_members(b);
  ck(cudaGraphLaunch(exec, b->stream), "cudaGraphLaunch");
  ck(cudaEventRecord(b->ev_flight, b->stream), "event");
  for (mcb200_ctx *c : b->m) ck(cudaStreamWaitEvent(c->stream, b->ev_flight, 0), "wait");
}

// One full timestep, replayed from (or first captured into) the graph of
// its (store parity, Poisson members).
template <typename R>
void batch_graph_step(mcb200_batch *b, uint64_t due) {
  const int n = (int)b->m.size();
  const std::pair<int, uint64_t> key{b->m[0]->cur, due};
  auto it = b->graphs.find(key);
  if (it == b->graphs.end()) {
    mcb200_batch::Graph g;
    std::vector<uint64_t> before(n);
    for (int k = 0; k < n; ++k) before[k] = b->m[k]->launches;
    const uint64_t batch_before = b->launches;
    cudaGraph_t graph = nullptr;
    ck(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeRelaxed), "cudaStreamBeginCapture");
    try {
      batch_full_step<R>(b, due);  // advances the host state by one step; the work runs at the launch below
    } catch (...) {
      cudaGraph_t broken = nullptr;
      cudaStreamEndCapture(b->stream, &broken);
      if (broken) cudaGraphDestroy(broken);
      throw;
    }
    ck(cudaStreamEndCapture(b->stream, &graph), "cudaStreamEndCapture");
    const cudaError_t e = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    ck(e, "cudaGraphInstantiate");
    g.member_launches.resize(n);
    for (int k = 0; k < n; ++k) g.member_launches[k] = b->m[k]->launches - before[k];
    g.batch_launches = b->launches - batch_before;
    launch_graph(b, g.exec);
    b->graphs.emplace(key, std::move(g));
    b->graph_captures += 1;
    return;
  }
  launch_graph(b, it->second.exec);
  // the host-side effects of the step the graph holds
  for (int k = 0; k < n; ++k) {
    mcb200_ctx *c = b->m[k];
    c->cur = 1 - c->cur;
    c->n_stale = true;
    c->launches += it->second.member_launches[k];
    if (b->cfg[k].self_consistent && c->device_set) c->fields_set = true;
  }
  b->launches += it->second.batch_launches;
  b->steps_done += 1;
  for (uint32_t &st : b->member_step) ++st;
  b->graph_replays += 1;
}

// All members' streams joined into the batch stream.
void join_members(mcb200_batch *b) {
  for (size_t k = 0; k < b->m.size(); ++k) {
    ck(cudaEventRecord(b->ev_member[k], b->m[k]->stream), "event");
    ck(cudaStreamWaitEvent(b->stream, b->ev_member[k], 0), "wait");
  }
}

}  // namespace
}  // namespace mcb200::eng

using namespace mcb200;
using namespace mcb200::eng;

extern "C" {

int mcb200_batch_create(mcb200_ctx *const *ctxs, const mcb200_batch_member *members, int n, mcb200_batch **out) {
  if (!out || !ctxs || !members || n < 1) return MCB200_ERR_ARG;
  *out = nullptr;
  if (n > kMaxBatch) return MCB200_ERR_CAPACITY;
  mcb200_batch *b = new mcb200_batch;
  *out = b;
  const mcb200_ctx *first = ctxs[0];
  if (!first || first->device < 0) return bfail(b, MCB200_ERR_STATE, "mcb200_batch_create: a member has no device");
  b->device = first->device;
  b->precision = first->precision;
  for (int k = 0; k < n; ++k) {
    mcb200_ctx *c = ctxs[k];
    if (!c || c->device != b->device || c->ts != first->ts)
      return bfail(b, MCB200_ERR_ARG, "mcb200_batch_create: members must share the device and the band tables "
                                      "(mcb200_create_alike)");
    if (c->precision != b->precision)
      return bfail(b, MCB200_ERR_ARG, "mcb200_batch_create: members must share the flight precision");
    if (!c->mesh_set || !c->cells_set)
      return bfail(b, MCB200_ERR_STATE, "mcb200_batch_create: every member needs its mesh and cells");
    for (int j = 0; j < k; ++j)
      if (ctxs[j] == c) return bfail(b, MCB200_ERR_ARG, "mcb200_batch_create: a context appears twice");
    b->m.push_back(c);
    b->cfg.push_back(members[k]);
  }
  try {
    ck(cudaSetDevice(b->device), "cudaSetDevice");
    ck(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    ck(cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking), "cudaStreamCreate");
    ck(cudaEventCreateWithFlags(&b->ev_side, cudaEventDisableTiming), "cudaEventCreate");
    ck(cudaEventCreateWithFlags(&b->ev_side0, cudaEventDisableTiming), "cudaEventCreate");
    ck(cudaEventCreateWithFlags(&b->ev_steps, cudaEventDisableTiming), "cudaEventCreate");
    ck(cudaEventCreateWithFlags(&b->ev_flight, cudaEventDisableTiming), "cudaEventCreate");
    ck(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming), "cudaEventCreate");
    ck(cudaEventCreateWithFlags(&b->ev_solved, cudaEventDisableTiming), "cudaEventCreate");
    b->ev_member.assign(n, nullptr);
    for (int k = 0; k < n; ++k) ck(cudaEventCreateWithFlags(&b->ev_member[k], cudaEventDisableTiming), "event");
    const size_t entry = b->precision == MCB200_FLIGHT_FP32 ? sizeof(BatchInstT<float>) : sizeof(BatchInstT<double>);
    ck(cudaMalloc(&b->tables, 6 * (size_t)n * entry), "cudaMalloc");
    ck(cudaMalloc(&b->steps, (size_t)n * sizeof(uint32_t)), "cudaMalloc");
    ck(cudaMalloc(&b->tickets, (2 + mcb200_ctx::kGenerations) * sizeof(unsigned int)), "cudaMalloc");
    std::vector<uint32_t> first_steps(n);
    for (int k = 0; k < n; ++k) first_steps[k] = members[k].first_step;
    b->member_step = first_steps;
    ck(cudaMemcpy(b->steps, first_steps.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice), "copy");
    b->snap.assign((size_t)n * kSnapBytes, 0);
    if (b->precision == MCB200_FLIGHT_FP32) build_tables<float>(b);
    else build_tables<double>(b);
  } catch (const std::exception &e) {
    return bfail(b, MCB200_ERR_CUDA, e.what());
  }
  return MCB200_OK;
}

void mcb200_batch_destroy(mcb200_batch *b) { delete b; }

const char *mcb200_batch_last_error(const mcb200_batch *b) { return b ? b->error.c_str() : "null batch"; }

int mcb200_batch_step(mcb200_batch *b) {
  if (!b) return MCB200_ERR_ARG;
  for (mcb200_ctx *c : b->m) {
    if (!c->fields_set) return bfail(b, MCB200_ERR_STATE, "mcb200_batch_step: a member has no fields");
    if (c->precision != b->precision)
      return bfail(b, MCB200_ERR_STATE, "mcb200_batch_step: a member changed its flight precision");
    if (c->overflow_pending) {
      c->overflow_pending = false;
      return bfail(b, MCB200_ERR_CAPACITY, "particle store of a member full: GENERATE copies were dropped");
    }
  }
  try {
    ck(cudaSetDevice(b->device), "cudaSetDevice");
    if (b->precision == MCB200_FLIGHT_FP32) {
      if (!tables_current(b)) build_tables<float>(b);
      batch_transport<float>(b);
    } else {
      if (!tables_current(b)) build_tables<double>(b);
      batch_transport<double>(b);
    }
    return MCB200_OK;
  } catch (const std::exception &e) {
    return bfail(b, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_batch_run(mcb200_batch *b, int steps) {
  if (!b || steps < 0) return MCB200_ERR_ARG;
  try {  // pending statistics joined outside any capture
    ck(cudaSetDevice(b->device), "cudaSetDevice");
    for (mcb200_ctx *c : b->m) join_stat(c);
  } catch (const std::exception &e) {
    return bfail(b, MCB200_ERR_CUDA, e.what());
  }
  for (size_t k = 0; k < b->m.size(); ++k) {
    mcb200_ctx *c = b->m[k];
    if (!c->fields_set && !(b->cfg[k].self_consistent && c->device_set))
      return bfail(b, MCB200_ERR_STATE, "mcb200_batch_run: a member has no fields");
    if (c->precision != b->precision)
      return bfail(b, MCB200_ERR_STATE, "mcb200_batch_run: a member changed its flight precision");
    if (c->overflow_pending) {
      c->overflow_pending = false;
      return bfail(b, MCB200_ERR_CAPACITY, "particle store of a member full: GENERATE copies were dropped");
    }
  }
  try {
    ck(cudaSetDevice(b->device), "cudaSetDevice");
    for (int s = 0; s < steps; ++s) {
      const uint64_t due = poisson_due(b);
      if (b->precision == MCB200_FLIGHT_FP32) {
        if (!tables_current(b)) build_tables<float>(b);
        if (b->use_graphs) batch_graph_step<float>(b, due);
        else batch_full_step<float>(b, due);
      } else {
        if (!tables_current(b)) build_tables<double>(b);
        if (b->use_graphs) batch_graph_step<double>(b, due);
        else batch_full_step<double>(b, due);
      }
    }
    return MCB200_OK;
  } catch (const std::exception &e) {
    return bfail(b, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_batch_autotune(mcb200_batch *b, int trial_steps, mcb200_batch_tuning *best) {
  if (!b || trial_steps < 1) return MCB200_ERR_ARG;
  static const int flight_blocks[] = {1, 2};
  static const int grid_per_sm[] = {2, 4, 8};
  static const int sort_buckets[] = {1, 2, 4, 8};
  mcb200_batch_tuning win{0, 0, 0, 1e300, 0, 0, 1, 0, 0, 0};
  int tried = 0;
  auto apply = [&](mcb200_batch_tuning &t) {
    b->blocks_per_sm = t.flight_blocks_per_sm;
    b->overlap = t.overlap != 0;
    b->pair_solves = t.pair_solves != 0;
    b->smem_table = t.smem_table != 0;
    for (mcb200_ctx *c : b->m) {
      c->grid_per_sm = t.grid_per_sm;
      mcb200_set_sort_bucket(c, t.sort_bucket);
    }
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    mcb200_batch_set_solo(b, t.solo_min_particles, &t.solo_members);
    b->drop_graphs();  // the graphs hold the previous launch shapes
  };
  // ms per step of one setting: one untimed step (it captures the graphs of
  // this setting), then the timed ones
  auto measure = [&](mcb200_batch_tuning &t, double &ms) -> int {
    apply(t);
    if (int rc = mcb200_batch_run(b, 1)) return rc;
    if (int rc = mcb200_batch_mark(b, 6)) return rc;
    if (int rc = mcb200_batch_run(b, trial_steps)) return rc;
    if (int rc = mcb200_batch_mark(b, 7)) return rc;
    if (int rc = mcb200_batch_elapsed_ms(b, 6, 7, &ms)) return rc;
    ms /= trial_steps;
    return MCB200_OK;
  };
  // The simulations change while they are timed (particle counts drift), so
  // the candidates of a stage are timed in order and again in reverse order
  // and each keeps the mean of its two times: a linear drift cancels.
  auto stage = [&](std::vector<mcb200_batch_tuning> &cands) -> int {
    std::vector<double> sum(cands.size(), 0.0);
    for (int pass = 0; pass < 2; ++pass)
      for (size_t i = 0; i < cands.size(); ++i) {
        const size_t j = pass == 0 ? i : cands.size() - 1 - i;
        double ms = 0;
        if (int rc = measure(cands[j], ms)) return rc;
        sum[j] += ms;
      }
    win.ms_per_step = 1e300;
    for (size_t i = 0; i < cands.size(); ++i)
      if (sum[i] / 2 < win.ms_per_step) {
        win = cands[i];
        win.ms_per_step = sum[i] / 2;
      }
    tried += (int)cands.size();
    return MCB200_OK;
  };
  const int overlap0 = b->overlap ? 1 : 0, pair0 = b->pair_solves ? 1 : 0;
  const int bucket0 = b->m.empty() ? 1 : mcb200_get_sort_bucket(b->m[0]), table0 = b->smem_table ? 1 : 0;
  const uint64_t solo0 = b->solo_min;
  std::vector<mcb200_batch_tuning> shapes;
  for (int fb : flight_blocks)
    for (int gs : grid_per_sm)
      shapes.push_back(mcb200_batch_tuning{fb, gs, overlap0, 0.0, 0, pair0, bucket0, table0, solo0, 0});
  if (int rc = stage(shapes)) return rc;
  std::vector<mcb200_batch_tuning> modes;  // overlap, pairing and the table's place, with the fastest shapes
  for (int v = 0; v < 8; ++v) {
    mcb200_batch_tuning t = win;
    t.overlap = v & 1 ? 1 - overlap0 : overlap0;
    t.pair_solves = v & 2 ? 1 - pair0 : pair0;
    t.smem_table = v & 4 ? 1 - table0 : table0;
    modes.push_back(t);
  }
  if (int rc = stage(modes)) return rc;
  std::vector<mcb200_batch_tuning> widths;  // sort-bucket widths, with the fastest of the above
  widths.push_back(win);
  for (int w : sort_buckets)
    if (w != win.sort_bucket) {
      mcb200_batch_tuning t = win;
      t.sort_bucket = w;
      widths.push_back(t);
    }
  if (int rc = stage(widths)) return rc;
  // members flying solo: none, all, or those above a quartile of the counts
  std::vector<uint64_t> counts;
  for (mcb200_ctx *c : b->m) counts.push_back(mcb200_num_particles(c));
  std::sort(counts.begin(), counts.end());
  std::vector<uint64_t> thresholds{0, 1};
  for (int q = 1; q <= 3; ++q) thresholds.push_back(std::max<uint64_t>(counts[counts.size() * q / 4], 1));
  std::sort(thresholds.begin(), thresholds.end());
  thresholds.erase(std::unique(thresholds.begin(), thresholds.end()), thresholds.end());
  std::vector<mcb200_batch_tuning> solos{win};
  for (uint64_t t : thresholds)
    if (t != win.solo_min_particles) {
      mcb200_batch_tuning c = win;
      c.solo_min_particles = t;
      solos.push_back(c);
    }
  if (int rc = stage(solos)) return rc;
  tried -= 3;  // each stage's first candidate is the previous stage's winner
  win.candidates = tried;
  apply(win);
  if (best) *best = win;
  return MCB200_OK;
}

int mcb200_batch_use_graphs(mcb200_batch *b, int enable) {
  if (!b) return MCB200_ERR_ARG;
  b->use_graphs = enable != 0;
  if (!b->use_graphs) {
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    b->drop_graphs();
  }
  return MCB200_OK;
}

int mcb200_batch_sync(mcb200_batch *b) {
  if (!b) return MCB200_ERR_ARG;
  try {
    ck(cudaSetDevice(b->device), "cudaSetDevice");
    ck(cudaStreamSynchronize(b->stream), "sync");
    for (mcb200_ctx *c : b->m) {
      ck(cudaStreamSynchronize(c->stream), "sync");
      pull_counts(c);
    }
    return MCB200_OK;
  } catch (const CapacityError &e) {
    return bfail(b, MCB200_ERR_CAPACITY, e.what());
  } catch (const std::exception &e) {
    return bfail(b, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_batch_set_grid(mcb200_batch *b, int blocks_per_sm) {
  if (!b || blocks_per_sm < 0 || blocks_per_sm > 8) return MCB200_ERR_ARG;
  b->blocks_per_sm = blocks_per_sm;
  return MCB200_OK;
}

int mcb200_batch_set_overlap(mcb200_batch *b, int enable) {
  if (!b) return MCB200_ERR_ARG;
  cudaSetDevice(b->device);
  cudaStreamSynchronize(b->stream);
  b->overlap = enable != 0;
  b->drop_graphs();
  return MCB200_OK;
}

int mcb200_batch_set_solo(mcb200_batch *b, uint64_t min_particles, int *members) {
  if (!b) return MCB200_ERR_ARG;
  try {
    ck(cudaSetDevice(b->device), "cudaSetDevice");
    ck(cudaStreamSynchronize(b->stream), "sync");
    uint64_t mask = 0;
    int count = 0;
    for (size_t k = 0; k < b->m.size(); ++k) {
      mcb200_ctx *c = b->m[k];
      ck(cudaStreamSynchronize(c->stream), "sync");
      pull_counts(c);
      if (min_particles > 0 && c->n >= min_particles) {
        mask |= 1ull << k;
        ++count;
      }
    }
    if (mask != b->solo) b->drop_graphs();
    b->solo = mask;
    b->solo_min = (size_t)min_particles;
    if (members) *members = count;
    return MCB200_OK;
  } catch (const CapacityError &e) {
    return bfail(b, MCB200_ERR_CAPACITY, e.what());
  } catch (const std::exception &e) {
    return bfail(b, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_batch_set_smem_table(mcb200_batch *b, int enable) {
  if (!b) return MCB200_ERR_ARG;
  cudaSetDevice(b->device);
  cudaStreamSynchronize(b->stream);
  b->smem_table = enable != 0;
  b->drop_graphs();
  return MCB200_OK;
}

int mcb200_batch_set_pairing(mcb200_batch *b, int enable) {
  if (!b) return MCB200_ERR_ARG;
  cudaSetDevice(b->device);
  cudaStreamSynchronize(b->stream);
  b->pair_solves = enable != 0;
  b->drop_graphs();
  return MCB200_OK;
}

int mcb200_batch_mark(mcb200_batch *b, int slot) {
  if (!b || slot < 0 || slot >= 8) return MCB200_ERR_ARG;
  try {
    ck(cudaSetDevice(b->device), "cudaSetDevice");
    if (!b->marks[slot]) ck(cudaEventCreate(&b->marks[slot]), "cudaEventCreate");
    join_members(b);
    ck(cudaEventRecord(b->marks[slot], b->stream), "cudaEventRecord");
    // members' later work follows the mark as well
    for (mcb200_ctx *c : b->m) ck(cudaStreamWaitEvent(c->stream, b->marks[slot], 0), "wait");
    return MCB200_OK;
  } catch (const std::exception &e) {
    return bfail(b, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_batch_elapsed_ms(mcb200_batch *b, int from, int to, double *ms) {
  if (!b || !ms || from < 0 || from >= 8 || to < 0 || to >= 8) return MCB200_ERR_ARG;
  if (!b->marks[from] || !b->marks[to]) return bfail(b, MCB200_ERR_STATE, "mark not recorded");
  try {
    ck(cudaSetDevice(b->device), "cudaSetDevice");
    ck(cudaEventSynchronize(b->marks[to]), "cudaEventSynchronize");
    float f = 0;
    ck(cudaEventElapsedTime(&f, b->marks[from], b->marks[to]), "cudaEventElapsedTime");
    *ms = f;
    return MCB200_OK;
  } catch (const std::exception &e) {
    return bfail(b, MCB200_ERR_CUDA, e.what());
  }
}

int mcb200_batch_info(const mcb200_batch *b, int *members, uint64_t *steps_done, uint64_t *launches,
                      uint64_t *graph_captures, uint64_t *graph_replays) {
  if (!b) return MCB200_ERR_ARG;
  if (members) *members = (int)b->m.size();
  if (steps_done) *steps_done = b->steps_done;
  if (launches) *launches = b->launches;
  if (graph_captures) *graph_captures = b->graph_captures;
  if (graph_replays) *graph_replays = b->graph_replays;
  return MCB200_OK;
}

}  // extern "C"
