// static_sort.cu -- counting sort of a caller-owned particle store by mesh
// cell, with no device allocation at all.
//
// For callers that cannot allocate device memory themselves or through us:
// a host framework that owns every device buffer and hands out slices of
// its own pool, code running where cudaMalloc would stall or serialise
// other work (a real-time loop, another library's allocator holding the
// device), or a plugin host that forbids allocation outside its own calls.
// They pass the input and output particle arrays; the sort's scratch (cell
// histogram, cell offsets, scan tile sums) lives in one file-scope device
// array that every GPU loading this library holds until process exit.
//
// The kernels are the ones mcb200_step uses for its sort (flight_kernels.cu);
// only the scratch differs.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "engine_kernels.h"
#include "mcb200.h"

using namespace mcb200;

namespace {

constexpr int kMaxCells = MCB200_STATIC_SORT_MAX_CELLS;
constexpr int kMaxTiles = (kMaxCells + 1023) / 1024;
// [0, kMaxCells) histogram, [kMaxCells, 2 kMaxCells) offsets,
// [2 kMaxCells, 2 kMaxCells + kMaxTiles) tile sums, then the total.
constexpr size_t kScratchWords = 2 * (size_t)kMaxCells + kMaxTiles + 1;

__device__ __align__(256) unsigned int g_sort_scratch[kScratchWords];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
unsigned int *g_scratch_addr[kMaxDevices] = {};
int g_sm_count[kMaxDevices] = {};

// Device address of g_sort_scratch on the current device.  In host code the
// symbol names a host-side stand-in, not device memory, so the address is
// looked up once per device with that device current and cached.
int scratch_for_current_device(unsigned int **addr, int *sms) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return MCB200_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_sort_scratch) != cudaSuccess || !p) return MCB200_ERR_CUDA;
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return MCB200_ERR_CUDA;
    g_scratch_addr[dev] = static_cast<unsigned int *>(p);
    g_sm_count[dev] = n;
  }
  *addr = g_scratch_addr[dev];
  *sms = g_sm_count[dev];
  return MCB200_OK;
}

DevParticles as_dev(const mcb200_device_particles &p) {
  DevParticles d;
  d.x = p.x; d.y = p.y; d.z = p.z;
  d.kx = p.kx; d.ky = p.ky; d.kz = p.kz;
  d.energy = p.energy; d.charge = p.charge;
  d.cell = p.cell; d.itet = p.itet; d.meta = p.meta; d.uid = p.uid;
  return d;
}

}  // namespace

extern "C" int mcb200_sort_particles_static(const mcb200_device_particles *in, size_t n, int nx, int ny, int nz,
                                            const mcb200_device_particles *out, size_t *n_out, void *stream) {
  if (!in || !out || nx <= 0 || ny <= 0 || nz <= 0 || nx > 1023 || ny > 1023 || nz > 1023) return MCB200_ERR_ARG;
  const long long cells = (long long)nx * ny * nz;
  if (cells > kMaxCells) return MCB200_ERR_CAPACITY;
  if (n > (size_t)0x7fffffff) return MCB200_ERR_CAPACITY;
  unsigned int *s = nullptr;
  int sms = 0;
  if (int rc = scratch_for_current_device(&s, &sms)) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  unsigned int *hist = s, *offsets = s + kMaxCells, *tiles = s + 2 * (size_t)kMaxCells, *total = tiles + kMaxTiles;
  const int grid = (int)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, (size_t)sms * 8));
  // launch_cell_sort clears the histogram before counting; offsets, tile sums
  // and the total are fully overwritten by the scan.
  launch_cell_sort(as_dev(*in), DevCount{nullptr, nullptr, (int)n}, as_dev(*out), (int)cells, nx, nz, hist, offsets,
                   tiles, total, grid, st);
  if (cudaGetLastError() != cudaSuccess) return MCB200_ERR_CUDA;
  if (n_out) {
    unsigned int kept = 0;
    if (cudaMemcpyAsync(&kept, total, sizeof(kept), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return MCB200_ERR_CUDA;
    *n_out = kept;
  }
  return MCB200_OK;
}
