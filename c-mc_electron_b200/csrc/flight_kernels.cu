// flight_kernels.cu -- free-flight kernels and the per-step particle
// bookkeeping (mid-step copies, removal of caught particles, counting sort
// by mesh cell).
//
// Step structure (replaces MeshQuantities::update_particle +
// local_migrate, src/mcmodel.cpp:1460-1505 and :1615-1638):
//   1. flight_kernel: every particle flies dt on its own random stream;
//      caught particles are marked dead in their meta word.
//   2. child_flight_kernel, repeated: copies made by GENERATE / GENREF fly
//      the rest of the step (they may make copies of their own).
//   3. append_children_kernel: surviving copies join the store with uids
//      next_uid + rank of (parent, sub).
//   4. cell_histogram / scan_tiles / cell_scatter: survivors and copies are
//      counting-sorted by cell into the second particle buffer; the
//      scatter's last block makes the sorted count the particle count.
#include <algorithm>

#include "engine_kernels.h"
#include "flight_physics.cuh"
#include "pdl.cuh"
#include "flight_physics_impl.cuh"

namespace mcb200 {

// Resident blocks of 256 threads per SM the flight kernels are compiled for
// (the register budget per thread follows: 2 -> 128, 3 -> 80).
#ifndef MCB200_FLIGHT_BLOCKS_F32
#define MCB200_FLIGHT_BLOCKS_F32 2
#endif
#ifndef MCB200_FLIGHT_BLOCKS_F64
#define MCB200_FLIGHT_BLOCKS_F64 2
#endif
template <typename R>
constexpr int kFlightBlocks = sizeof(R) == 4 ? MCB200_FLIGHT_BLOCKS_F32 : MCB200_FLIGHT_BLOCKS_F64;
// Threads per block of the flight kernels (a tuning define like the above).
#ifndef MCB200_FLIGHT_THREADS
#define MCB200_FLIGHT_THREADS 256
#endif
constexpr int kFlightThreads = MCB200_FLIGHT_THREADS;

constexpr uint32_t kMetaDead = 1u << 16;
constexpr uint32_t kMetaUnfinished = 1u << 17;

template <typename R>
__device__ void load_sym(SymSmemT<R> &S, const DevTables &T) {
  for (int i = threadIdx.x; i < 48 * 6; i += blockDim.x) S.symi[i] = T.symi[i];
  for (int i = threadIdx.x; i < 5 * 48; i += blockDim.x) S.newisym[i] = T.newisym[i];
  for (int i = threadIdx.x; i < 3 * 5 * 48; i += blockDim.x) S.bz[i] = (R)T.bz[i];
  for (int i = threadIdx.x; i < 3 * 48; i += blockDim.x) S.refl[i] = T.reflect_isym[i];
  __syncthreads();
}

// Loading and storing the flown particles of the main store (StoreIO) and
// of a child generation (ChildIO).
template <typename R>
struct StoreIO {
  DevParticlesT<R> P;
  double dt;
  uint32_t step;  // the particles' step number (their random streams)
  __device__ bool load(int p, FlyerT<R> &f) const {
    const uint32_t meta = P.meta[p];
    if (meta & kMetaDead) return false;
    f.step_ = step;
    f.x = P.x[p]; f.y = P.y[p]; f.z = P.z[p];
    f.kx = P.kx[p]; f.ky = P.ky[p]; f.kz = P.kz[p];
    f.energy = P.energy[p];
    f.charge = P.charge[p];
    const uint32_t c = P.cell[p];
    f.ic = c & 1023; f.jc = (c >> 10) & 1023; f.kc = (c >> 20) & 1023;
    f.itet = P.itet[p];
    f.isym = meta & 255;
    f.type = (meta >> 8) & 255;
    f.start_stream(P.uid[p], 0);
    f.nchild = 0;
    f.left_time = dt;
    return true;
  }
  __device__ void store(int p, const FlyerT<R> &f, int r) const {
    P.x[p] = f.x; P.y[p] = f.y; P.z[p] = f.z;
    P.kx[p] = f.kx; P.ky[p] = f.ky; P.kz[p] = f.kz;
    P.energy[p] = f.energy;
    P.cell[p] = pack_cell(f.ic, f.jc, f.kc);
    P.itet[p] = f.itet;
    uint32_t m = (uint32_t)f.isym | ((uint32_t)f.type << 8);
    if (r == 1) m |= kMetaDead;
    if (r == 2) m |= kMetaUnfinished;
    P.meta[p] = m;
  }
};
template <typename R>
struct ChildIO {
  DevChildrenT<R> C;
  uint32_t step;
  __device__ bool load(int p, FlyerT<R> &f) const {
    f.step_ = step;
    f.x = C.x[p]; f.y = C.y[p]; f.z = C.z[p];
    f.kx = C.kx[p]; f.ky = C.ky[p]; f.kz = C.kz[p];
    f.energy = C.energy[p];
    f.charge = C.charge[p];
    const uint32_t c = C.cell[p];
    f.ic = c & 1023; f.jc = (c >> 10) & 1023; f.kc = (c >> 20) & 1023;
    f.itet = C.itet[p];
    f.isym = C.meta[p] & 255;
    f.type = (C.meta[p] >> 8) & 255;
    f.start_stream(C.parent_uid[p], C.sub[p]);
    f.nchild = 0;
    f.left_time = C.left_time[p];
    return true;
  }
  __device__ void store(int p, const FlyerT<R> &f, int r) const {
    C.x[p] = f.x; C.y[p] = f.y; C.z[p] = f.z;
    C.kx[p] = f.kx; C.ky[p] = f.ky; C.kz[p] = f.kz;
    C.energy[p] = f.energy;
    C.cell[p] = pack_cell(f.ic, f.jc, f.kc);
    C.itet[p] = f.itet;
    uint32_t m = (uint32_t)f.isym | ((uint32_t)f.type << 8);
    if (r == 1) m |= kMetaDead;
    if (r == 2) m |= kMetaUnfinished;
    C.meta[p] = m;
  }
};

// Persistent flight: each lane holds one particle at a time and advances it
// one event per pass; a lane whose particle has finished its step stores it
// and takes the next particle index from `ticket` (one atomic per warp for
// all lanes that need work).  Lanes therefore stay busy while the warp's
// other particles finish, instead of idling until the slowest one is done.
// Every particle's draws come from its own stream, so the result does not
// depend on which lane flies it or when.
//
// kLaneEvents (launches of one simulation): the event count of each finished
// particle is summed in the lane and the warp adds its total to the
// simulation's counter once, at the end, instead of one atomic on that one
// address per particle.  A batched launch counts per particle (its particles
// belong to different simulations).
template <typename R, bool kLaneEvents, class IO>
__device__ __forceinline__ void fly_interleaved(const FlightCtxT<R> &F, const SymSmemT<R> &S, const IO &io, int n,
                                                unsigned int *ticket) {
  FlyerT<R> f(F, S);
  const unsigned lane = threadIdx.x & 31u;
  int p = -1;
  bool exhausted = false;
  uint32_t events = 0;  // < 2^31 + kMaxEvents: flushed whenever it passes 2^31
  auto done = [&]() {
    const int r = f.template finish<!kLaneEvents>();
    if constexpr (kLaneEvents) {
      events += (uint32_t)f.loop;
      if (events >= 0x80000000u) {
        atomicAdd(&F.Y.counters[kCntEvents], (unsigned long long)events);
        events = 0;
      }
    }
    return r;
  };
  for (;;) {
    if (!exhausted) {
      const unsigned need = __ballot_sync(0xffffffffu, p < 0);
      if (need) {
        const int leader = __ffs(need) - 1;
        unsigned base = 0;
        if ((int)lane == leader) base = atomicAdd(ticket, (unsigned)__popc(need));
        base = __shfl_sync(0xffffffffu, base, leader);
        if ((unsigned long long)base + __popc(need) >= (unsigned long long)n) exhausted = true;
        if (p < 0) {
          const unsigned q = base + __popc(need & ((1u << lane) - 1u));
          if (q < (unsigned)n && io.load((int)q, f)) {
            p = (int)q;
            f.begin();
            if (!(f.left_time > 0)) {
              io.store(p, f, done());
              p = -1;
            }
          }
        }
      }
    }
    if (!__any_sync(0xffffffffu, p >= 0)) {
      if (exhausted) break;
      continue;
    }
    if (p >= 0 && f.iterate()) {
      io.store(p, f, done());
      p = -1;
    }
  }
  if constexpr (kLaneEvents) {
    unsigned long long sum = events;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, off);
    if (lane == 0 && sum) atomicAdd(&F.Y.counters[kCntEvents], sum);
  }
}

template <typename R>
__global__ void __launch_bounds__(kFlightThreads, kFlightBlocks<R>) flight_kernel(FlightCtxT<R> F, DevParticlesT<R> P,
                                                                       DevCount n, unsigned int *ticket) {
  __shared__ SymSmemT<R> S;
  load_sym(S, F.T);  // the band tables: nothing the kernel ahead writes
  pdl_wait();
  const int count = n.get();
  if (count == 0) return;
  const uint32_t step = F.step_dev ? *F.step_dev : F.step;
  fly_interleaved<R, true>(F, S, StoreIO<R>{P, F.dt, step}, count, ticket);
}

// Copies made during the previous pass (buffer `in`) fly the rest of their
// step; copies they make go to `F.C`.
template <typename R>
__global__ void __launch_bounds__(kFlightThreads, kFlightBlocks<R>) child_flight_kernel(FlightCtxT<R> F, DevChildrenT<R> in,
                                                              unsigned int *ticket) {
  pdl_wait();
  const int count = min((int)*in.count, in.capacity);
  if (count == 0) return;
  __shared__ SymSmemT<R> S;
  load_sym(S, F.T);
  const uint32_t step = F.step_dev ? *F.step_dev : F.step;
  fly_interleaved<R, true>(F, S, ChildIO<R>{in, step}, count, ticket);
}

// ---- batched flight ------------------------------------------------------
// Many simulations in one persistent launch.  Each block copies the batch's
// table of simulations (BatchInstT, one per simulation) into shared memory
// and forms the prefix of their particle counts, read on the device; a lane
// that takes ticket q flies particle q - prefix[k] of simulation k, the
// largest k with prefix[k] <= q, with that simulation's mesh, fields,
// tallies, copy buffer, dt, seed and step (FlyerT::I).  A particle's draws
// still come from its own stream (seed, uid, step), so it flies exactly as
// in a launch of its simulation alone.
template <typename R, bool kChild>
struct BatchIO {
  const BatchInstT<R> *I;  // shared memory
  const int *prefix;       // [ninst + 1], shared memory
  int ninst;
  __device__ __forceinline__ int find(int q) const {
    int lo = 0, hi = ninst - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (prefix[mid] <= q) lo = mid;
      else hi = mid - 1;
    }
    return lo;
  }
  __device__ bool load(int q, FlyerT<R> &f) const {
    const int k = find(q);
    const BatchInstT<R> &b = I[k];
    f.I = &b;
    const int p = q - prefix[k];
    if constexpr (kChild) return ChildIO<R>{b.in, b.step}.load(p, f);
    else return StoreIO<R>{b.P, b.dt, b.step}.load(p, f);
  }
  __device__ void store(int q, const FlyerT<R> &f, int r) const {
    const BatchInstT<R> *b = static_cast<const BatchInstT<R> *>(f.I);
    const int p = q - prefix[b - I];
    if constexpr (kChild) ChildIO<R>{b->in, b->step}.store(p, f, r);
    else StoreIO<R>{b->P, b->dt, b->step}.store(p, f, r);
  }
};

// Dynamic shared memory of a batched launch over `ninst` simulations: the
// table of simulations (when it is copied there) and the prefix of their
// particle counts.
template <typename R>
constexpr size_t batch_smem_bytes(int ninst, bool table) {
  return (table ? (size_t)ninst * sizeof(BatchInstT<R>) : 0) + (size_t)(ninst + 1) * sizeof(int);
}

// F holds the band tables (its per-simulation part is unused); steps[k] is
// simulation k's step number (device memory, advanced between steps).
// Simulations whose bit in `members` is clear contribute no particles.
// kSmemTable: every block copies the table into shared memory (about 0.8 KB
// per simulation, taken from the SM's L1 share) and takes the step numbers
// from `steps`; otherwise lanes read the table where it lies (global memory,
// through L1), whose step fields advance_batch_steps keeps current.
template <typename R, bool kChild, bool kSmemTable>
__global__ void __launch_bounds__(kFlightThreads, kFlightBlocks<R>) batch_flight_kernel(const __grid_constant__ FlightCtxT<R> F,
                                                                             const BatchInstT<R> *inst,
                                                                             int ninst, uint64_t members,
                                                                             const uint32_t *steps,
                                                                             unsigned int *ticket) {
  extern __shared__ __align__(16) unsigned char batch_smem[];
  __shared__ SymSmemT<R> S;
  const BatchInstT<R> *I;
  int *prefix;
  if constexpr (kSmemTable) {
    BatchInstT<R> *T = reinterpret_cast<BatchInstT<R> *>(batch_smem);
    prefix = reinterpret_cast<int *>(T + ninst);
    static_assert(sizeof(BatchInstT<R>) % 8 == 0, "the table is copied in 8-byte words");
    const unsigned long long *src = reinterpret_cast<const unsigned long long *>(inst);
    unsigned long long *dst = reinterpret_cast<unsigned long long *>(T);
    const int words = ninst * (int)(sizeof(BatchInstT<R>) / 8);
    for (int w = threadIdx.x; w < words; w += blockDim.x) dst[w] = src[w];
    __syncthreads();
    if (threadIdx.x == 0)
      for (int k = 0; k < ninst; ++k) T[k].step = steps[k];
    I = T;
  } else {
    prefix = reinterpret_cast<int *>(batch_smem);
    I = inst;
  }
  if (threadIdx.x == 0) {
    int run = 0;
    for (int k = 0; k < ninst; ++k) {
      prefix[k] = run;
      if ((members >> k) & 1ull)
        run += kChild ? min((int)*I[k].in.count, I[k].in.capacity) : min((int)*I[k].n, I[k].capacity);
    }
    prefix[ninst] = run;
  }
  load_sym(S, F.T);  // ends with a barrier: the table and prefix are visible
  const int total = prefix[ninst];
  if (total == 0) return;
  fly_interleaved<R, false>(F, S, BatchIO<R, kChild>{I, prefix, ninst}, total, ticket);
}

// Step numbers of a batch: steps[k] += 1, and the step field of simulation
// k in each of the `ntab` tables of n simulations.
template <typename R>
__global__ void advance_batch_steps(uint32_t *steps, BatchInstT<R> *tab, int n, int ntab) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const uint32_t v = steps[k] + 1;
  steps[k] = v;
  for (int t = 0; t < ntab; ++t) tab[(size_t)t * n + k].step = v;
}
template <typename R>
void launch_advance_batch_steps(uint32_t *steps, BatchInstT<R> *tab, int n, int ntab, cudaStream_t s) {
  advance_batch_steps<R><<<(n + 63) / 64, 64, 0, s>>>(steps, tab, n, ntab);
}

// FP32 flight's per-cell records (DevMesh::cell32): the fields in float and
// the Brooks-Herring factors of GetImpScRate / GetImpScGamma /
// EleImpScUpdateK (src/ElectronImpurityScatter.cpp:6-306) evaluated once per
// cell in FP64 from the cell's screening density and doping.
//
// The step's counters are reset in the same launch (block 0: zeroed work
// tickets, copy counts and appended count), which the flight then reads.
__device__ __forceinline__ void reset_step_counters(const StepCounters &z, int t) {
  if (t < 1 + kChildGenerations) {
    z.tickets[t] = 0u;
    *z.count[t] = 0u;
  }
  if (t == 0) *z.appended = 0u;
}
__global__ void cell_records32_kernel(DevTables T, DevMesh M, float4 *out, int cells, StepCounters z) {
  pdl_wait();
  if (blockIdx.x == 0) reset_step_counters(z, threadIdx.x);
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cells) return;
  const double rho = M.rho[c], da = M.da[c];
  const bool on = (da * T.conc0 >= 1e22) && !(M.surface_scatter && M.surface_impurity && M.in_surf[c]);
  const double eebeta = T.frickel * 4 * kPiD * rho / (2.0 * T.meld * T.eps_si);
  const double fr = T.frickel * rho;
  const float bh_a = on ? (float)(da * T.meld * sqrt(2.0 * T.meld) / (kPiD * (fr * fr))) : 0.0f;
  const float bh_b = on ? (float)(4.0 * T.melt / (eebeta * T.meld)) : 0.0f;
  const double *e = M.efield + 3 * (size_t)c, *h = M.hfield + 3 * (size_t)c;
  out[3 * (size_t)c + 0] = make_float4((float)e[0], (float)e[1], (float)e[2], bh_a);
  out[3 * (size_t)c + 1] = make_float4((float)h[0], (float)h[1], (float)h[2], bh_b);
  out[3 * (size_t)c + 2] = make_float4((float)(T.frickel * 4 * kPiD * rho / (8.0 * T.melt * T.eps_si)),
                                       (float)(T.frickel * 4 * kPiD * rho / T.eps_si), (float)(0.120 / T.eV0), 0.0f);
}

// ---- counting sort by cell ------------------------------------------------
__device__ __forceinline__ int cell_linear(uint32_t c, int nx, int nz) {
  return (int)((((c >> 10) & 1023) * nx + (c & 1023)) * nz + ((c >> 20) & 1023));
}

// Buckets of 2^shift consecutive cells of the linear order (z fastest):
// shift 0 sorts by cell; wider buckets make the histogram and its scan
// shorter and leave the particles of a bucket in arrival order.  When the
// scatter will compute the sorted store's charge bounds, they start from
// zero here.
__global__ void cell_histogram(const uint32_t *cell, const uint32_t *meta, DevCount count, int nx, int nz,
                               unsigned int *hist, int shift, unsigned long long *bounds) {
  pdl_wait();
  const int n = count.get();
  if (bounds && blockIdx.x == 0 && threadIdx.x < 4) bounds[threadIdx.x] = 0ull;
  // a warp walks 32 consecutive particles; lanes of the same bucket (a
  // cell-sorted store holds runs of them) add their count with one atomic
  const unsigned lane = threadIdx.x & 31u;
  for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += gridDim.x * blockDim.x) {
    const int p = base + (int)lane;
    unsigned int key = 0xffffffffu;
    if (p < n && !(meta[p] & kMetaDead)) key = (unsigned int)(cell_linear(cell[p], nx, nz) >> shift);
    const unsigned int peers = __match_any_sync(0xffffffffu, key);
    if (key != 0xffffffffu && (int)lane == __ffs(peers) - 1) atomicAdd(&hist[key], (unsigned int)__popc(peers));
  }
}

// Exclusive scan of `count` values, single pass per 1024-wide tile plus a
// tile-sum pass (cells are at most ~10^6, so three small launches suffice).
// Exclusive scan of the tile sums in place by one block of 1024 threads,
// 1024 tiles per pass with the running total carried between passes.
__device__ void scan_tile_sums_block(unsigned int *tile_sums, int ntiles, unsigned int *total) {
  __shared__ unsigned int s[1024];
  unsigned int carry = 0;
  for (int base = 0; base < ntiles; base += 1024) {
    const int t = base + threadIdx.x;
    const unsigned int v = t < ntiles ? __ldcg(tile_sums + t) : 0u;  // written by other blocks: read at L2
    s[threadIdx.x] = v;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
      const unsigned int a = threadIdx.x >= (unsigned)off ? s[threadIdx.x - off] : 0u;
      __syncthreads();
      s[threadIdx.x] += a;
      __syncthreads();
    }
    if (t < ntiles) tile_sums[t] = carry + s[threadIdx.x] - v;
    carry += s[1023];
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

// Exclusive scan of each 1024-wide tile, and its sum into tile_sums.  With
// `blocks` (a counter that is zero between launches) the last block to
// finish then scans the tile sums too (scan_tile_sums' work, one launch
// fewer).  clear (or null): the input, zeroed once read (the step's sort
// keeps its histogram zero between sorts, so no memset precedes it).
__global__ void scan_tiles(const unsigned int *in, unsigned int *out, unsigned int *tile_sums, int n,
                           unsigned int *blocks, unsigned int *total, unsigned int *clear) {
  __shared__ unsigned int s[1024];
  __shared__ bool last;
  pdl_wait();
  const int i = blockIdx.x * 1024 + threadIdx.x;
  const unsigned int v = i < n ? in[i] : 0u;
  if (clear && i < n) clear[i] = 0u;
  s[threadIdx.x] = v;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    unsigned int t = threadIdx.x >= (unsigned)off ? s[threadIdx.x - off] : 0u;
    __syncthreads();
    s[threadIdx.x] += t;
    __syncthreads();
  }
  if (i < n) out[i] = s[threadIdx.x] - v;
  if (threadIdx.x == 1023) tile_sums[blockIdx.x] = s[1023];
  if (blocks == nullptr) return;  // uniform over the grid
  if (threadIdx.x == 1023) {
    __threadfence();
    last = atomicAdd(blocks, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;  // uniform over the block
  __threadfence();
  scan_tile_sums_block(tile_sums, (int)gridDim.x, total);
  if (threadIdx.x == 0) *blocks = 0u;
}
__global__ void scan_tile_sums(unsigned int *tile_sums, int ntiles, unsigned int *total) {
  scan_tile_sums_block(tile_sums, ntiles, total);
}
__global__ void scan_add(unsigned int *out, const unsigned int *tile_sums, int n) {
  const int i = blockIdx.x * 1024 + threadIdx.x;
  if (i < n) out[i] += tile_sums[blockIdx.x];
}

// bounds (optional, zeroed by the histogram): the sorted store's charge
// bounds in charge_bounds_kernel's layout, {max |q| bits of electrons, of
// holes, electron count, hole count}, from the particles this pass moves.
// finish (optional): the end of the step, by the grid's last block to
// finish (every block has read the count by then).
// tile_base (optional): cursor holds tile-local offsets and the tile's
// exclusive prefix is added (scan_add's work, one launch fewer; the cursor
// then ends as tile-local cell ends).
template <typename R>
__global__ void __launch_bounds__(256) cell_scatter(DevParticlesT<R> src, DevCount count, DevParticlesT<R> dst,
                                                    unsigned int *cursor, int nx, int nz, int shift,
                                                    unsigned long long *bounds, StepFinish finish,
                                                    const unsigned int *tile_base) {
  pdl_wait();
  const int n = count.get();
  unsigned long long mx[2] = {0, 0}, cnt[2] = {0, 0};
  // lanes of the same bucket take consecutive slots with one atomic
  const unsigned lane = threadIdx.x & 31u;
  for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += gridDim.x * blockDim.x) {
    const int p = base + (int)lane;
    const uint32_t m = p < n ? src.meta[p] : kMetaDead;
    const bool live = !(m & kMetaDead);
    const unsigned int key = live ? (unsigned int)(cell_linear(src.cell[p], nx, nz) >> shift) : 0xffffffffu;
    const unsigned int peers = __match_any_sync(0xffffffffu, key);
    const int leader = __ffs(peers) - 1;
    unsigned int first = 0;
    if (live && (int)lane == leader) first = atomicAdd(&cursor[key], (unsigned int)__popc(peers));
    first = __shfl_sync(0xffffffffu, first, leader);
    if (!live) continue;
    const unsigned int q = first + (unsigned int)__popc(peers & ((1u << lane) - 1u)) +
                           (tile_base ? tile_base[key >> 10] : 0u);
    const double charge = src.charge[p];
    dst.x[q] = src.x[p]; dst.y[q] = src.y[p]; dst.z[q] = src.z[p];
    dst.kx[q] = src.kx[p]; dst.ky[q] = src.ky[p]; dst.kz[q] = src.kz[p];
    dst.energy[q] = src.energy[p]; dst.charge[q] = charge;
    dst.cell[q] = src.cell[p];
    dst.itet[q] = src.itet[p];
    dst.meta[q] = m & 0xffffu;
    dst.uid[q] = src.uid[p];
    const int t = ((m >> 8) & 255) == 0 ? 0 : 1;
    const unsigned long long b = (unsigned long long)__double_as_longlong(fabs(charge));
    mx[t] = b > mx[t] ? b : mx[t];
    cnt[t] += 1;
  }
  if (bounds != nullptr) {  // uniform over the grid
    __shared__ unsigned long long red[4][8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int t = 0; t < 2; ++t) {
      for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long om = __shfl_down_sync(0xffffffffu, mx[t], o);
        mx[t] = om > mx[t] ? om : mx[t];
        cnt[t] += __shfl_down_sync(0xffffffffu, cnt[t], o);
      }
      if (lane == 0) {
        red[t][warp] = mx[t];
        red[2 + t][warp] = cnt[t];
      }
    }
    __syncthreads();
    if (threadIdx.x < 4) {
      const int v = threadIdx.x;
      unsigned long long a = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) a = v < 2 ? (red[v][w] > a ? red[v][w] : a) : a + red[v][w];
      if (v < 2) {
        if (a) atomicMax(bounds + v, a);
      } else if (a) {
        atomicAdd(bounds + v, a);
      }
    }
  }
  if (finish.n != nullptr) {  // uniform over the grid
    __syncthreads();  // every thread of the block has read the count
    if (threadIdx.x == 0) {
      __threadfence();
      const unsigned int done = atomicAdd(finish.blocks, 1u);
      if (done == gridDim.x - 1) {  // the last block: every block has read the count
        __threadfence();
        *finish.particle_steps += *finish.n;
        *finish.n = *finish.sorted_total;
        *finish.next_uid += *finish.appended;
        *finish.blocks = 0u;
      }
    }
  }
}

// The surviving copies of every generation (already flown) join the store
// after its *n particles, in one launch.  A copy's uid is *next_uid + the
// number of surviving copies with a smaller (parent uid, sub) key, over all
// generations (the key set is the concatenation of the generations).  A
// block ranks 32 copies at a time, one a lane: the keys of all copies are
// staged through shared memory in chunks, each of the eight warps counts
// the smaller live keys of every eighth one (a broadcast read per compare),
// and the eight counts of a lane are added.  The place in the store is
// taken from `appended` (order does not matter: the cell sort follows); a
// copy that would land beyond the store's capacity is dropped and raises
// *overflow (the host reports it).
template <typename R>
struct CopyRef {
  const ChildSetT<R> &set;
  int cnt[kChildGenerations];
  __device__ explicit CopyRef(const ChildSetT<R> &s) : set(s) {
#pragma unroll
    for (int q = 0; q < kChildGenerations; ++q) cnt[q] = min((int)*set.g[q].count, set.g[q].capacity);
  }
  // generation and index of copy i of the concatenation
  __device__ __forceinline__ void locate(int i, int &gen, int &local) const {
    gen = 0;
    local = i;
#pragma unroll
    for (int q = 0; q + 1 < kChildGenerations; ++q)
      if (gen == q && local >= cnt[q]) {
        local -= cnt[q];
        ++gen;
      }
  }
  __device__ __forceinline__ void key(int i, uint64_t &k, bool &alive) const {
    int gen, local;
    locate(i, gen, local);
    const DevChildrenT<R> &c = set.g[gen];
    k = ((uint64_t)c.parent_uid[local] << 32) | c.sub[local];
    alive = !(c.meta[local] & kMetaDead);
  }
};

template <typename R>
__global__ void __launch_bounds__(256) append_children_kernel(ChildSetT<R> set, const unsigned int *next_uid,
                                                              DevParticlesT<R> dst, const unsigned int *n,
                                                              int capacity, unsigned int *appended,
                                                              unsigned int *overflow) {
  constexpr int kChunk = 2048;
  __shared__ uint64_t keys[kChunk];
  __shared__ uint32_t part[8][32];
  pdl_wait();
  const CopyRef<R> ref(set);
  int total = 0;
#pragma unroll
  for (int q = 0; q < kChildGenerations; ++q) total += ref.cnt[q];
  if (total == 0) return;
  const uint32_t uid0 = *next_uid;
  const unsigned int n0 = *n;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int base_i = blockIdx.x * 32; base_i < total; base_i += gridDim.x * 32) {
    const int i = base_i + lane;
    uint64_t my = ~0ull;
    bool my_alive = false;
    if (i < total) ref.key(i, my, my_alive);
    uint32_t rank = 0;
    for (int base = 0; base < total; base += kChunk) {
      const int m = min(kChunk, total - base);
      __syncthreads();  // the previous chunk (and the previous group's counts) are consumed
      for (int j = threadIdx.x; j < m; j += 256) {
        uint64_t kj;
        bool aj;
        ref.key(base + j, kj, aj);
        keys[j] = aj ? kj : ~0ull;  // a dead copy ranks after every live one
      }
      __syncthreads();
      for (int q = warp; q < m; q += 8) rank += keys[q] < my ? 1u : 0u;
    }
    part[warp][lane] = rank;
    __syncthreads();
    if (warp == 0 && i < total && my_alive) {
      uint32_t r = 0;
#pragma unroll
      for (int w = 0; w < 8; ++w) r += part[w][lane];
      int gen, local;
      ref.locate(i, gen, local);
      const DevChildrenT<R> &c = set.g[gen];
      const unsigned long long q = (unsigned long long)n0 + atomicAdd(appended, 1u);
      if (q >= (unsigned long long)capacity) {
        *overflow = 1u;
      } else {
        dst.x[q] = c.x[local]; dst.y[q] = c.y[local]; dst.z[q] = c.z[local];
        dst.kx[q] = c.kx[local]; dst.ky[q] = c.ky[local]; dst.kz[q] = c.kz[local];
        dst.energy[q] = c.energy[local]; dst.charge[q] = c.charge[local];
        dst.cell[q] = c.cell[local];
        dst.itet[q] = c.itet[local];
        dst.meta[q] = c.meta[local] & 0xffffu;
        dst.uid[q] = uid0 + r;
      }
    }
  }
}

// ---- initial ensemble ---------------------------------------------------------
// New particle q (uid = uid0 + q) of carrier `type` in cell cell_of[q]:
// position uniform in the cell (init_particle_data,
// src/particle_init.cpp:185-207) and k-state from select_kstate
// (src/mcmodel.cpp:3006-3057): energy from the Boltzmann distribution,
// accepted against the DOS, band by the DOS share, k uniform on the
// iso-energy surface.  Draws: stream (seed, uid, kSeedStreamStep, 0).
// The sampling runs in FP64 for both stores, so an FP32 store starts from
// the same ensemble as an FP64 one (rounded once, positions made
// cell-relative).

template <typename R>
__global__ void __launch_bounds__(256) seed_kernel(FlightCtx F, DevParticlesT<R> P, int offset, int n,
                                                   const int *cell_of, const double *charge, int type,
                                                   uint32_t uid0) {
  __shared__ SymSmem S;
  load_sym(S, F.T);
  const DevTables &T = F.T;
  const double tmp_const = 1 - exp(-T.emax);
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    Flyer f(F, S);
    const int c = cell_of[q];
    const int kc = c % F.M.nz, ic = (c / F.M.nz) % F.M.nx, jc = c / (F.M.nz * F.M.nx);
    f.ic = ic; f.jc = jc; f.kc = kc;
    f.type = type;
    f.start_stream(uid0 + q, 0);
    double lamda = f.Random();
    f.x = lamda * F.M.lx[ic] + (1 - lamda) * F.M.lx[ic + 1];
    lamda = f.Random();
    f.y = lamda * F.M.ly[jc] + (1 - lamda) * F.M.ly[jc + 1];
    lamda = f.Random();
    f.z = lamda * F.M.lz[kc] + (1 - lamda) * F.M.lz[kc + 1];
    f.itet = 0;
    f.kx = f.ky = f.kz = 0;
    bool ok = false;
    for (int attempt = 0; attempt < 100000 && !ok; ++attempt) {
      f.energy = -log(1 - f.Random() * tmp_const);
      // CALDOSSUM (src/Band.cpp:2267-2295) and CALDOS (:2234-2264)
      const TabPos p = tab_pos(T, f.energy);
      const double ddos = tab_at_strided(T.sumdos + type, 3, p);
      double rdos = f.Random() * T.dosmax[type];
      if (rdos > ddos) continue;
      for (f.iband = T.bandof[type]; f.iband < T.bandof[type] + T.nband[type]; f.iband++) {
        rdos -= tab_at(T.dos + (size_t)f.iband * kNT, p);
        if (rdos < 0) break;
      }
      f.isym = ((int)(f.Random() * 48)) % 48;
      if (f.iband >= T.bandof[type] + T.nband[type]) continue;  // rounding left no band: draw again
      f.get_state();
      if (f.self) continue;
      ok = true;
    }
    if (!ok) count(F.Y, kCntNoTet);
    const int o = offset + q;
    if constexpr (FlightReal<R>::kCellRelative) {
      P.x[o] = (R)(f.x - F.M.lx[ic]); P.y[o] = (R)(f.y - F.M.ly[jc]); P.z[o] = (R)(f.z - F.M.lz[kc]);
    } else {
      P.x[o] = f.x; P.y[o] = f.y; P.z[o] = f.z;
    }
    P.kx[o] = (R)f.kx; P.ky[o] = (R)f.ky; P.kz[o] = (R)f.kz;
    P.energy[o] = f.energy;
    P.charge[o] = charge[q];
    P.cell[o] = pack_cell(ic, jc, kc);
    P.itet[o] = f.itet;
    P.meta[o] = (uint32_t)f.isym | ((uint32_t)type << 8) | (ok ? 0u : kMetaDead);
    P.uid[o] = f.uid;
  }
}

// ---- host-side launchers ----------------------------------------------------
template <typename R>
void launch_seed(const FlightCtx &F, const DevParticlesT<R> &P, int offset, int n, const int *cell_of,
                 const double *charge, int type, uint32_t uid0, int grid, cudaStream_t s) {
  if (n > 0) seed_kernel<R><<<grid, 256, 0, s>>>(F, P, offset, n, cell_of, charge, type, uid0);
}
// Blocks of the persistent flight kernels: enough to fill every SM at the
// kernel's occupancy, fewer when there are fewer particles than threads.
// Launch settings are looked up once per device (the current device at the
// launch) and kept: a process may drive several GPUs.
constexpr int kMaxDevices = 64;
inline int current_device() {
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= kMaxDevices) d = 0;
  return d;
}
template <typename R>
int flight_grid(int n, int block, int sm_count) {
  static int per_sm_of[kMaxDevices] = {};
  int &per_sm = per_sm_of[current_device()];
  if (per_sm == 0) {
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, flight_kernel<R>, block, 0) != cudaSuccess || b < 1) b = 1;
    per_sm = b;
  }
  const long long want = ((long long)n + block - 1) / block;
  return (int)std::max<long long>(1, std::min<long long>(want, (long long)per_sm * sm_count));
}

template <typename R>
void launch_flight(const FlightCtxT<R> &F, const DevParticlesT<R> &P, DevCount n, unsigned int *ticket, int sm_count,
                   cudaStream_t s) {
  launch_pdl(flight_kernel<R>, flight_grid<R>(n.max, kFlightThreads, sm_count), kFlightThreads, 0, s, F, P, n, ticket);
}
template <typename R>
void launch_child_flight(const FlightCtxT<R> &F, const DevChildrenT<R> &in, int n_hint, unsigned int *ticket,
                         int sm_count, cudaStream_t s) {
  // One block per SM: a step's copies are few (their lanes refill from the
  // same counter however many there are), and most generations are empty.
  const int n = (int)std::min<long long>(n_hint, (long long)sm_count * kFlightThreads);
  launch_pdl(child_flight_kernel<R>, flight_grid<R>(n, kFlightThreads, sm_count), kFlightThreads, 0, s, F, in, ticket);
}
template <typename R>
int launch_batch_flight(const FlightCtxT<R> &F, const BatchInstT<R> *inst, int ninst, uint64_t members,
                        const uint32_t *steps, bool child, unsigned int *ticket, int blocks_per_sm, int sm_count,
                        cudaStream_t s, bool smem_table) {
  if (ninst < 1 || ninst > kMaxBatch) return 1;
  const size_t smem = batch_smem_bytes<R>(ninst, smem_table);
  auto kernel = smem_table ? (child ? batch_flight_kernel<R, true, true> : batch_flight_kernel<R, false, true>)
                           : (child ? batch_flight_kernel<R, true, false> : batch_flight_kernel<R, false, false>);
  if (smem_table) {
    // the opt-in to more than 48 KB of dynamic shared memory holds per device
    static bool opted[kMaxDevices][2] = {};
    bool &done = opted[current_device()][child ? 1 : 0];
    if (!done) {
      if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)batch_smem_bytes<R>(kMaxBatch, true)) != cudaSuccess)
        return 1;
      done = true;
    }
  }
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kFlightThreads, smem) != cudaSuccess ||
      per_sm < 1)
    return 1;
  if (blocks_per_sm > 0) per_sm = std::min(per_sm, blocks_per_sm);
  kernel<<<per_sm * sm_count, kFlightThreads, smem, s>>>(F, inst, ninst, members, steps, ticket);
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
}
void launch_records_and_reset(const DevTables &T, const DevMesh &M, float4 *out, int cells, const StepCounters &z,
                              cudaStream_t s) {
  launch_pdl(cell_records32_kernel, std::max((cells + 255) / 256, 1), 256, 0, s, T, M, out, cells, z);
}
template <typename R>
void launch_append_children(const ChildSetT<R> &set, unsigned int *next_uid, const DevParticlesT<R> &dst,
                            const unsigned int *n, int capacity, unsigned int *appended, unsigned int *overflow,
                            int grid, cudaStream_t s) {
  launch_pdl(append_children_kernel<R>, grid, 256, 0, s, set, next_uid, dst, n, capacity, appended, overflow);
}
__global__ void step_reset_kernel(StepCounters z) { reset_step_counters(z, threadIdx.x); }
void launch_step_reset(const StepCounters &z, cudaStream_t s) { step_reset_kernel<<<1, 32, 0, s>>>(z); }
void launch_exclusive_scan(const unsigned int *in, unsigned int *out, unsigned int *tile_sums, unsigned int *total,
                           int n, cudaStream_t s) {
  const int tiles = (n + 1023) / 1024;
  scan_tiles<<<tiles, 1024, 0, s>>>(in, out, tile_sums, n, nullptr, nullptr, nullptr);
  scan_tile_sums<<<1, 1024, 0, s>>>(tile_sums, tiles, total);
  scan_add<<<tiles, 1024, 0, s>>>(out, tile_sums, n);
}
template <typename R>
void launch_cell_sort(const DevParticlesT<R> &src, DevCount n, const DevParticlesT<R> &dst, int ncells, int nx,
                      int nz, unsigned int *hist, unsigned int *offsets, unsigned int *tile_sums, unsigned int *total,
                      int shift, unsigned long long *bounds, int grid, cudaStream_t s, const StepFinish &finish) {
  const int buckets = (ncells + (1 << shift) - 1) >> shift;
  const int tiles = (buckets + 1023) / 1024;
  if (finish.n != nullptr) {
    // the step's sort: the histogram starts from the zeros the last one
    // left, the tile sums are scanned by scan_tiles' last block (which also
    // clears the histogram), the tile prefixes added by the scatter, the
    // step ended by its last block
    launch_pdl(cell_histogram, grid, 256, 0, s, src.cell, src.meta, n, nx, nz, hist, shift, bounds);
    launch_pdl(scan_tiles, tiles, 1024, 0, s, (const unsigned int *)hist, offsets, tile_sums, buckets,
               finish.scan_blocks, total, hist);
    launch_pdl(cell_scatter<R>, grid, 256, 0, s, src, n, dst, offsets, nx, nz, shift, bounds, finish, tile_sums);
    return;
  }
  cudaMemsetAsync(hist, 0, sizeof(unsigned int) * buckets, s);
  cell_histogram<<<grid, 256, 0, s>>>(src.cell, src.meta, n, nx, nz, hist, shift, bounds);
  scan_tiles<<<tiles, 1024, 0, s>>>(hist, offsets, tile_sums, buckets, nullptr, nullptr, nullptr);
  scan_tile_sums<<<1, 1024, 0, s>>>(tile_sums, tiles, total);
  scan_add<<<tiles, 1024, 0, s>>>(offsets, tile_sums, buckets);
  cell_scatter<R><<<grid, 256, 0, s>>>(src, n, dst, offsets, nx, nz, shift, bounds, finish, nullptr);
}

#define MCB200_INSTANTIATE(R)                                                                                   \
  template void launch_seed<R>(const FlightCtx &, const DevParticlesT<R> &, int, int, const int *,            \
                               const double *, int, uint32_t, int, cudaStream_t);                             \
  template void launch_flight<R>(const FlightCtxT<R> &, const DevParticlesT<R> &, DevCount, unsigned int *, int, \
                                 cudaStream_t);                                                                 \
  template void launch_child_flight<R>(const FlightCtxT<R> &, const DevChildrenT<R> &, int, unsigned int *, int, \
                                       cudaStream_t);                                                           \
  template void launch_append_children<R>(const ChildSetT<R> &, unsigned int *, const DevParticlesT<R> &,     \
                                          const unsigned int *, int, unsigned int *, unsigned int *, int,       \
                                          cudaStream_t);                                                        \
  template int launch_batch_flight<R>(const FlightCtxT<R> &, const BatchInstT<R> *, int, uint64_t,             \
                                      const uint32_t *, bool, unsigned int *, int, int, cudaStream_t, bool);    \
  template void launch_advance_batch_steps<R>(uint32_t *, BatchInstT<R> *, int, int, cudaStream_t);           \
  template void launch_cell_sort<R>(const DevParticlesT<R> &, DevCount, const DevParticlesT<R> &, int, int, int, \
                                    unsigned int *, unsigned int *, unsigned int *, unsigned int *, int,        \
                                    unsigned long long *, int, cudaStream_t, const StepFinish &);
MCB200_INSTANTIATE(double)
MCB200_INSTANTIATE(float)
#undef MCB200_INSTANTIATE

}  // namespace mcb200
