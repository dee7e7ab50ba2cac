// engine_kernels.h -- launchers shared between the engine translation units.
#pragma once

#include <cuda_runtime.h>

#include "device_state.cuh"

namespace mcb200 {

struct FlightCtx;

void launch_flight(const FlightCtx &F, const DevParticles &P, int n, int grid, int block, cudaStream_t s);
void launch_child_flight(const FlightCtx &F, const DevChildren &in, int grid, int block, cudaStream_t s);
void launch_child_keys(const DevChildren &c, int n, uint64_t *keys, uint8_t *alive, cudaStream_t s);
void launch_child_rank(const uint64_t *keys, const uint8_t *alive, int n, uint32_t next_uid, uint32_t *uid_out,
                       cudaStream_t s);
void launch_children_to_particles(const DevChildren &c, int n, const uint32_t *uids, const uint8_t *alive,
                                  const DevParticles &dst, int dst_offset, unsigned int *dst_count, cudaStream_t s);
void launch_seed(const FlightCtx &F, const DevParticles &P, int offset, int n, const int *cell_of,
                 const double *charge, int type, uint32_t uid0, int grid, cudaStream_t s);
void launch_exclusive_scan(const unsigned int *in, unsigned int *out, unsigned int *tile_sums, unsigned int *total,
                           int n, cudaStream_t s);
void launch_cell_sort(const DevParticles &src, int n, const DevParticles &dst, int ncells, int nx, int nz,
                      unsigned int *hist, unsigned int *offsets, unsigned int *tile_sums, unsigned int *total,
                      int grid, cudaStream_t s);

}  // namespace mcb200
