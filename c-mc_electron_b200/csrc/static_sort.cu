// static_sort.cu -- counting sort of a caller-owned particle store by mesh
// cell, with no device allocation at all.
//
// For callers that cannot allocate device memory themselves or through us:
// a host framework that owns every device buffer and hands out slices of
// its own pool, code running where cudaMalloc would stall or serialise
// other work (a real-time loop, another library's allocator holding the
// device), or a plugin host that forbids allocation outside its own calls.
// They pass the input and output particle arrays; the sort's scratch (cell
// histogram, cell offsets, scan tile sums, the kept count and a range-error
// word) lives in one file-scope device array that every GPU loading this
// library holds until process exit.
//
// The sort is the one mcb200_step runs after each flight (histogram, scan,
// scatter).  The engine trusts its own cell indices; a caller's may be
// wrong, so the histogram and scatter here skip any live particle whose
// cell lies outside the mesh and raise the error word instead of touching
// memory past the histogram or the output arrays.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>

#include "engine_kernels.h"
#include "mcb200.h"

using namespace mcb200;

namespace {

constexpr int kMaxCells = MCB200_STATIC_SORT_MAX_CELLS;
constexpr int kMaxTiles = (kMaxCells + 1023) / 1024;
// [0, kMaxCells) histogram, [kMaxCells, 2 kMaxCells) offsets,
// [2 kMaxCells, 2 kMaxCells + kMaxTiles) tile sums, then the kept count and
// the range-error word (adjacent: one 8-byte read returns both).
constexpr size_t kTotalWord = 2 * (size_t)kMaxCells + kMaxTiles;
constexpr size_t kScratchWords = kTotalWord + 2;
static_assert(kTotalWord % 2 == 0, "the count and the error word share one aligned 8-byte read");

__device__ __align__(256) unsigned int g_sort_scratch[kScratchWords];

constexpr uint32_t kDead = 1u << 16;

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

// Linear cell of a packed i | j << 10 | k << 20 cell, or -1 outside the mesh.
__device__ __forceinline__ int checked_linear(uint32_t c, int nx, int ny, int nz) {
  const int i = (int)(c & 1023u), j = (int)((c >> 10) & 1023u), k = (int)((c >> 20) & 1023u);
  if (i >= nx || j >= ny || k >= nz) return -1;
  return (j * nx + i) * nz + k;
}

__global__ void checked_histogram(const uint32_t *cell, const uint32_t *meta, int n, int nx, int ny, int nz,
                                  unsigned int *hist, unsigned int *bad) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    if (meta[p] & kDead) continue;
    const int lin = checked_linear(cell[p], nx, ny, nz);
    if (lin < 0) {
      atomicOr(bad, 1u);
      continue;
    }
    atomicAdd(&hist[lin], 1u);
  }
}

__global__ void checked_scatter(DevParticles src, int n, DevParticles dst, unsigned int *cursor, int nx, int ny,
                                int nz) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const uint32_t m = src.meta[p];
    if (m & kDead) continue;
    const int lin = checked_linear(src.cell[p], nx, ny, nz);
    if (lin < 0) continue;
    const unsigned int q = atomicAdd(&cursor[lin], 1u);
    dst.x[q] = src.x[p]; dst.y[q] = src.y[p]; dst.z[q] = src.z[p];
    dst.kx[q] = src.kx[p]; dst.ky[q] = src.ky[p]; dst.kz[q] = src.kz[p];
    dst.energy[q] = src.energy[p]; dst.charge[q] = src.charge[p];
    dst.cell[q] = src.cell[p];
    dst.itet[q] = src.itet[p];
    dst.meta[q] = m & 0xffffu;
    dst.uid[q] = src.uid[p];
  }
}

DevParticles as_dev(const mcb200_device_particles &p) {
  DevParticles d;
  d.x = p.x; d.y = p.y; d.z = p.z;
  d.kx = p.kx; d.ky = p.ky; d.kz = p.kz;
  d.energy = p.energy; d.charge = p.charge;
  d.cell = p.cell; d.itet = p.itet; d.meta = p.meta; d.uid = p.uid;
  return d;
}

// The byte ranges [begin, end) of the twelve arrays of a store of n particles.
void ranges(const mcb200_device_particles &p, size_t n, uintptr_t lo[12], uintptr_t hi[12], bool *null_field) {
  const void *ptr[12] = {p.x, p.y, p.z, p.kx, p.ky, p.kz, p.energy, p.charge, p.cell, p.itet, p.meta, p.uid};
  const size_t width[12] = {8, 8, 8, 8, 8, 8, 8, 8, 4, 4, 4, 4};
  *null_field = false;
  for (int f = 0; f < 12; ++f) {
    if (!ptr[f]) *null_field = true;
    lo[f] = reinterpret_cast<uintptr_t>(ptr[f]);
    hi[f] = lo[f] + width[f] * n;
  }
}

// True when any input array shares bytes with any output array (the scatter
// reads the input while other threads write the output).
bool in_out_overlap(const mcb200_device_particles &in, const mcb200_device_particles &out, size_t n, bool *null_field) {
  uintptr_t ilo[12], ihi[12], olo[12], ohi[12];
  bool ni = false, no = false;
  ranges(in, n, ilo, ihi, &ni);
  ranges(out, n, olo, ohi, &no);
  *null_field = ni || no;
  if (n == 0) return false;
  for (int a = 0; a < 12; ++a)
    for (int b = 0; b < 12; ++b)
      if (ilo[a] < ohi[b] && olo[b] < ihi[a]) return true;
  return false;
}

}  // namespace

extern "C" int mcb200_sort_particles_static(const mcb200_device_particles *in, size_t n, int nx, int ny, int nz,
                                            const mcb200_device_particles *out, size_t *n_out, void *stream) {
  if (!in || !out || nx <= 0 || ny <= 0 || nz <= 0 || nx > 1023 || ny > 1023 || nz > 1023) return MCB200_ERR_ARG;
  const long long cells = (long long)nx * ny * nz;
  if (cells > kMaxCells) return MCB200_ERR_CAPACITY;
  if (n > (size_t)0x7fffffff) return MCB200_ERR_CAPACITY;
  bool null_field = false;
  if (in_out_overlap(*in, *out, n, &null_field) || (n > 0 && null_field)) return MCB200_ERR_ARG;
  // An error left pending by the caller's earlier work is the caller's: leave
  // it in place and do nothing, rather than clear it or take it for ours.
  if (cudaPeekAtLastError() != cudaSuccess) return MCB200_ERR_CUDA;
  unsigned int *s = nullptr;
  int sms = 0;
  if (int rc = scratch_for_current_device(&s, &sms)) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  unsigned int *hist = s, *offsets = s + kMaxCells, *tiles = s + 2 * (size_t)kMaxCells, *total = s + kTotalWord,
               *bad = total + 1;
  const int grid = (int)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, (size_t)sms * 8));
  // The previous call's contents stay in the array: the histogram and the
  // error word start from zero here; offsets, tile sums and the kept count
  // are fully overwritten by the scan.
  if (cudaMemsetAsync(hist, 0, sizeof(unsigned int) * (size_t)cells, st) != cudaSuccess ||
      cudaMemsetAsync(bad, 0, sizeof(unsigned int), st) != cudaSuccess)
    return MCB200_ERR_CUDA;
  const DevParticles src = as_dev(*in), dst = as_dev(*out);
  checked_histogram<<<grid, 256, 0, st>>>(src.cell, src.meta, (int)n, nx, ny, nz, hist, bad);
  launch_exclusive_scan(hist, offsets, tiles, total, (int)cells, st);
  checked_scatter<<<grid, 256, 0, st>>>(src, (int)n, dst, offsets, nx, ny, nz);
  if (cudaGetLastError() != cudaSuccess) return MCB200_ERR_CUDA;
  // The kept count and the range check come back together; the call returns
  // once the sort has finished.
  unsigned int back[2] = {0, 0};
  if (cudaMemcpyAsync(back, total, sizeof(back), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return MCB200_ERR_CUDA;
  if (n_out) *n_out = back[0];
  return back[1] ? MCB200_ERR_ARG : MCB200_OK;
}
