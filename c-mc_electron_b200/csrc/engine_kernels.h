// engine_kernels.h -- launchers shared between the engine translation units.
// Templates over the flight precision R are instantiated for double (plain
// FP64 path) and float (FP32 flight) in flight_kernels.cu.
#pragma once

#include <cuda_runtime.h>

#include "device_state.cuh"

namespace mcb200 {

template <typename R>
struct FlightCtxT;
using FlightCtx = FlightCtxT<double>;

// Persistent flight launches: `ticket` is a zeroed device counter the blocks
// take particle indices from; the main flight reads its particle count from
// device memory (n.max sizes the grid), a child generation its own count;
// n_hint bounds the copies a generation holds.
template <typename R>
void launch_flight(const FlightCtxT<R> &F, const DevParticlesT<R> &P, DevCount n, unsigned int *ticket, int sm_count,
                   cudaStream_t s);
template <typename R>
void launch_child_flight(const FlightCtxT<R> &F, const DevChildrenT<R> &in, int n_hint, unsigned int *ticket,
                         int sm_count, cudaStream_t s);
// One persistent launch flying the particles (child == false) or the copies
// of one generation (child == true) of the simulations k < ninst with bit k
// of `members` set (inst: device table of BatchInstT, steps: their step
// numbers); blocks_per_sm <= 0: as many as fit.  Returns 0 on success.
template <typename R>
struct BatchInstT;
template <typename R>
int launch_batch_flight(const FlightCtxT<R> &F, const BatchInstT<R> *inst, int ninst, uint64_t members,
                        const uint32_t *steps, bool child, unsigned int *ticket, int blocks_per_sm, int sm_count,
                        cudaStream_t s, bool smem_table);
// steps[k] += 1 and the step field of simulation k in `ntab` consecutive
// tables of n simulations (the tables the batched flights read in place).
template <typename R>
void launch_advance_batch_steps(uint32_t *steps, BatchInstT<R> *tab, int n, int ntab, cudaStream_t s);

// The step's surviving copies (all generations) ranked by (parent uid, sub),
// given uids from *next_uid on, and appended to `dst` after its *n
// particles, in one launch; *appended (zeroed by the step reset) counts them,
// *overflow is set if the store is full.
template <typename R>
void launch_append_children(const ChildSetT<R> &set, unsigned int *next_uid, const DevParticlesT<R> &dst,
                            const unsigned int *n, int capacity, unsigned int *appended, unsigned int *overflow,
                            int grid, cudaStream_t s);
// The counters a step starts from, zeroed in one launch: the flight tickets,
// the copy count of every generation and of the sink, and the appended count.
struct StepCounters {
  unsigned int *tickets;  // [1 + kChildGenerations]
  unsigned int *count[kChildGenerations + 1];
  unsigned int *appended;  // copies appended to the store this step
};
void launch_step_reset(const StepCounters &z, cudaStream_t s);
// FP32 flight's per-cell records (DevMesh::cell32), [cells][3] float4, and
// the step reset of z, in one launch.
void launch_records_and_reset(const DevTables &T, const DevMesh &M, float4 *out, int cells, const StepCounters &z,
                              cudaStream_t s);
// The end of a step, done by the last block of the sort's scatter (n null:
// none): *particle_steps += *n; *n = *sorted_total; *next_uid += *appended.
// blocks, scan_blocks: counters that are zero between launches.  A sort
// with a StepFinish leaves `offsets` as tile-local cell ends (nothing reads
// them after the step's sort) and `hist` zero, and expects it zero (the
// refresh's sort, without one, zeroes it first and the refresh zeroes it
// again when done).
struct StepFinish {
  unsigned int *n = nullptr;
  const unsigned int *sorted_total = nullptr;
  unsigned int *next_uid = nullptr;
  const unsigned int *appended = nullptr;
  unsigned long long *particle_steps = nullptr;
  unsigned int *blocks = nullptr;
  unsigned int *scan_blocks = nullptr;
};
template <typename R>
void launch_seed(const FlightCtx &F, const DevParticlesT<R> &P, int offset, int n, const int *cell_of,
                 const double *charge, int type, uint32_t uid0, int grid, cudaStream_t s);
void launch_exclusive_scan(const unsigned int *in, unsigned int *out, unsigned int *tile_sums, unsigned int *total,
                           int n, cudaStream_t s);
// Counting sort of the live particles among the first n (device count) of
// `src` by cell into `dst`; *total = live particles, offsets = cell starts
// (after the scatter: cell ends).  With shift > 0 the keys are buckets of
// 2^shift consecutive cells (hist and offsets per bucket).  bounds (or
// null): the sorted store's charge bounds, as launch_charge_bounds writes.
template <typename R>
void launch_cell_sort(const DevParticlesT<R> &src, DevCount n, const DevParticlesT<R> &dst, int ncells, int nx,
                      int nz, unsigned int *hist, unsigned int *offsets, unsigned int *tile_sums, unsigned int *total,
                      int shift, unsigned long long *bounds, int grid, cudaStream_t s,
                      const StepFinish &finish = StepFinish{});

}  // namespace mcb200
