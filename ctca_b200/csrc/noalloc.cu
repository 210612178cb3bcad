// noalloc.cu -- particle compaction for callers that cannot allocate device
// memory.
//
// Some hosts of this library cannot call cudaMalloc: a Fortran code whose
// device arrays all come from its own memory manager (OpenACC / CUDA Fortran
// pools with a fixed budget), or a code that runs this step from inside a
// region where its framework forbids allocation.  emsesg_compact_noalloc
// drops particles with nid == -1 from a device buffer the caller owns,
// writing the survivors (in buffer order) into a second buffer the caller
// owns, and allocates nothing: its scratch (per-particle offsets and per-tile
// sums) is a file-scope __device__ array of fixed size, so every GPU that
// loads the library keeps it (about 4 MB) until the process exits.
//
// The scratch is shared by every call on a device and keeps the last call's
// contents.  Every entry a call reads is written by the same call first, so
// nothing has to start at zero.  Two calls whose kernels overlap on the GPU
// (different streams, or different host threads) use the same scratch and
// race: the caller must order them, e.g. on one stream.  The input, the
// output and the survivor count must not share a byte (EMSESG_ERR_ARG).
#include <mutex>

#include "common.cuh"

namespace {

constexpr int NA_TILE_THREADS = 1024;
constexpr int NA_ITEMS = 4;
constexpr int NA_TILE = NA_TILE_THREADS * NA_ITEMS;
constexpr int64_t NA_MAX = EMSESG_NOALLOC_MAX_PARTICLES;
constexpr int64_t NA_TILES = (NA_MAX + NA_TILE - 1) / NA_TILE;  // 256

// [0, NA_MAX): exclusive offset of each particle within its tile;
// [NA_MAX, NA_MAX + NA_TILES): tile totals, then their exclusive prefix.
static __device__ __align__(256) uint32_t g_compact_scratch[NA_MAX + NA_TILES];

// Tile pass: live flags and their exclusive prefix within each 4096-particle
// tile; the tile total goes to tile_sum[b].
__global__ void __launch_bounds__(NA_TILE_THREADS) k_na_tile(const emsesg_particle* __restrict__ in, int64_t n,
                                                              uint32_t* __restrict__ local,
                                                              uint32_t* __restrict__ tile_sum) {
  __shared__ uint32_t warp_sums[NA_TILE_THREADS / 32];
  int64_t base = (int64_t)blockIdx.x * NA_TILE + (int64_t)threadIdx.x * NA_ITEMS;
  uint32_t f[NA_ITEMS];
  uint32_t s = 0;
#pragma unroll
  for (int i = 0; i < NA_ITEMS; i++) {
    f[i] = (base + i < n && in[base + i].nid != -1) ? 1u : 0u;
    s += f[i];
  }
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t incl = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warp_sums[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = warp_sums[lane], wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += t;
    }
    warp_sums[lane] = wi - w;
    if (lane == 31) tile_sum[blockIdx.x] = wi;
  }
  __syncthreads();
  uint32_t run = warp_sums[warp] + incl - s;
#pragma unroll
  for (int i = 0; i < NA_ITEMS; i++) {
    if (base + i < n) local[base + i] = run;
    run += f[i];
  }
}

// One block: exclusive prefix of the (at most 256) tile totals, in place;
// the grand total is the number of survivors.
__global__ void k_na_tiles(uint32_t* tile_sum, int ntiles, int64_t* kept) {
  __shared__ uint32_t s[NA_TILES];
  int t = threadIdx.x;
  s[t] = t < ntiles ? tile_sum[t] : 0u;
  __syncthreads();
  for (int o = 1; o < (int)NA_TILES; o <<= 1) {
    uint32_t v = t >= o ? s[t - o] : 0u;
    __syncthreads();
    s[t] += v;
    __syncthreads();
  }
  if (t < ntiles) tile_sum[t] = t == 0 ? 0u : s[t - 1];
  if (t == NA_TILES - 1) *kept = (int64_t)s[t];
}

__global__ void k_na_scatter(const emsesg_particle* __restrict__ in, int64_t n, const uint32_t* __restrict__ local,
                             const uint32_t* __restrict__ tile_sum, emsesg_particle* __restrict__ out) {
  int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  if (in[m].nid != -1) out[tile_sum[m / NA_TILE] + local[m]] = in[m];
}

// Device address of the scratch per device.  Host code may not use the
// symbol itself as a device pointer.  Outside a stream capture every call
// looks the address up again (cheap), so a device reset, after which the
// module is loaded anew, leaves no stale pointer; inside a capture the address
// of the last call outside it is used.
constexpr int NA_MAX_DEVICES = 64;
uint32_t* g_scratch_ptr[NA_MAX_DEVICES] = {nullptr};
std::mutex g_scratch_mu;

int scratch_for_current_device(cudaStream_t st, uint32_t** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NA_MAX_DEVICES) return EMSESG_ERR_CUDA;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) return EMSESG_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (cap == cudaStreamCaptureStatusNone) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_compact_scratch) != cudaSuccess || !p) return EMSESG_ERR_CUDA;
    g_scratch_ptr[dev] = (uint32_t*)p;
  }
  if (!g_scratch_ptr[dev]) return EMSESG_ERR_CUDA;  // first call on this device inside a capture
  *out = g_scratch_ptr[dev];
  return EMSESG_OK;
}

// [a, a + na) and [b, b + nb) share a byte.
bool overlap(const void* a, size_t na, const void* b, size_t nb) {
  const uintptr_t x = (uintptr_t)a, y = (uintptr_t)b;
  return na > 0 && nb > 0 && x < y + nb && y < x + na;
}

}  // namespace

extern "C" int emsesg_compact_noalloc(const emsesg_particle* d_in, int64_t n, emsesg_particle* d_out,
                                      int64_t* d_kept, void* stream) {
  if (n < 0 || n > NA_MAX || (n > 0 && (!d_in || !d_out)) || !d_kept) return EMSESG_ERR_ARG;
  const size_t bytes = (size_t)n * sizeof(emsesg_particle);
  if (overlap(d_in, bytes, d_out, bytes) || overlap(d_kept, sizeof(int64_t), d_in, bytes) ||
      overlap(d_kept, sizeof(int64_t), d_out, bytes))
    return EMSESG_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  uint32_t* scratch = nullptr;
  int rc = scratch_for_current_device(st, &scratch);
  if (rc) return rc;
  uint32_t* local = scratch;
  uint32_t* tile_sum = scratch + NA_MAX;
  int ntiles = (int)((n + NA_TILE - 1) / NA_TILE);
  // Each launch reports its own status; an error left pending by earlier
  // work of the caller is neither cleared nor reported here.
  if (ntiles > 0) {
    void* args[] = {(void*)&d_in, (void*)&n, (void*)&local, (void*)&tile_sum};
    if (cudaLaunchKernel((const void*)k_na_tile, dim3(ntiles), dim3(NA_TILE_THREADS), args, 0, st) != cudaSuccess)
      return EMSESG_ERR_CUDA;
  }
  {
    void* args[] = {(void*)&tile_sum, (void*)&ntiles, (void*)&d_kept};
    if (cudaLaunchKernel((const void*)k_na_tiles, dim3(1), dim3((unsigned)NA_TILES), args, 0, st) != cudaSuccess)
      return EMSESG_ERR_CUDA;
  }
  if (n > 0) {
    void* args[] = {(void*)&d_in, (void*)&n, (void*)&local, (void*)&tile_sum, (void*)&d_out};
    if (cudaLaunchKernel((const void*)k_na_scatter, dim3((unsigned)((n + 255) / 256)), dim3(256), args, 0, st) !=
        cudaSuccess)
      return EMSESG_ERR_CUDA;
  }
  return EMSESG_OK;
}
