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
// take particle indices from; n_hint bounds the children a generation holds.
template <typename R>
void launch_flight(const FlightCtxT<R> &F, const DevParticlesT<R> &P, int n, unsigned int *ticket, int sm_count,
                   cudaStream_t s);
template <typename R>
void launch_child_flight(const FlightCtxT<R> &F, const DevChildrenT<R> &in, int n_hint, unsigned int *ticket,
                         int sm_count, cudaStream_t s);
// FP32 flight's per-cell records (DevMesh::cell32), [cells][3] float4.
void launch_cell_records32(const DevTables &T, const DevMesh &M, float4 *out, int cells, cudaStream_t s);
template <typename R>
void launch_child_keys(const DevChildrenT<R> &c, int n, uint64_t *keys, uint8_t *alive, cudaStream_t s);
void launch_child_rank(const uint64_t *keys, const uint8_t *alive, int n, uint32_t next_uid, uint32_t *uid_out,
                       cudaStream_t s);
template <typename R>
void launch_children_to_particles(const DevChildrenT<R> &c, int n, const uint32_t *uids, const uint8_t *alive,
                                  const DevParticlesT<R> &dst, int dst_offset, unsigned int *dst_count,
                                  cudaStream_t s);
template <typename R>
void launch_seed(const FlightCtx &F, const DevParticlesT<R> &P, int offset, int n, const int *cell_of,
                 const double *charge, int type, uint32_t uid0, int grid, cudaStream_t s);
void launch_exclusive_scan(const unsigned int *in, unsigned int *out, unsigned int *tile_sums, unsigned int *total,
                           int n, cudaStream_t s);
template <typename R>
void launch_cell_sort(const DevParticlesT<R> &src, int n, const DevParticlesT<R> &dst, int ncells, int nx, int nz,
                      unsigned int *hist, unsigned int *offsets, unsigned int *tile_sums, unsigned int *total,
                      int grid, cudaStream_t s);

}  // namespace mcb200
