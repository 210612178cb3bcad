// sort.cu -- device primitives of the cell sort and the compaction: an
// exclusive prefix sum and a stable LSD radix sort of (uint32 key, uint32
// value) pairs with 8-bit digits.
//
// Radix pass (reduce-then-scan):
//   1. k_radix_hist: every block counts the digits of its 4096-key tile;
//      counts go to hist[digit * nblocks + block].
//   2. exclusive scan of hist (digit-major), giving every (digit, block) its
//      first output slot.
//   3. k_radix_scatter: every warp ranks its 512 keys item by item with
//      __match_any_sync (stable within the warp), warps are offset by an
//      exclusive scan of their per-digit counts, and each key goes to
//      hist[digit, block] + warp offset + rank.  Ties keep input order, so
//      the pass (and the sort) is stable.
#include <algorithm>

#include "common.cuh"

namespace emsesg {

namespace {

constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

constexpr int RADIX = 256;
constexpr int SORT_THREADS = 256;
constexpr int SORT_WARPS = SORT_THREADS / 32;
constexpr int SORT_ITEMS = 16;
constexpr int SORT_TILE = SORT_THREADS * SORT_ITEMS;

// In-place exclusive scan of one 4096-element tile; tile total -> part[b].
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_tile(uint32_t* data, int64_t n, uint32_t* part) {
  __shared__ uint32_t warp_sums[SCAN_THREADS / 32];
  int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
  uint32_t v[SCAN_ITEMS];
  uint32_t s = 0;
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; i++) {
    v[i] = (base + i < n) ? data[base + i] : 0u;
    s += v[i];
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
    uint32_t w = warp_sums[lane];
    uint32_t wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += t;
    }
    warp_sums[lane] = wi - w;  // exclusive
    if (lane == 31 && part) part[blockIdx.x] = wi;
  }
  __syncthreads();
  uint32_t run = warp_sums[warp] + incl - s;
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; i++) {
    if (base + i < n) data[base + i] = run;
    run += v[i];
  }
}

__global__ void k_scan_add(uint32_t* data, int64_t n, const uint32_t* part) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  data[i] += part[i / SCAN_TILE];
}

__global__ void k_copy_u32(uint32_t* dst, const uint32_t* src) { *dst = *src; }

__global__ void __launch_bounds__(SORT_THREADS) k_radix_hist(const uint32_t* __restrict__ keys, int64_t n, int shift,
                                                             uint32_t* hist, int nblocks) {
  __shared__ uint32_t cnt[RADIX];
  cnt[threadIdx.x] = 0;
  __syncthreads();
  int64_t base = (int64_t)blockIdx.x * SORT_TILE;
#pragma unroll 4
  for (int it = 0; it < SORT_ITEMS; it++) {
    int64_t idx = base + (int64_t)it * SORT_THREADS + threadIdx.x;
    if (idx < n) atomicAdd(&cnt[(keys[idx] >> shift) & (RADIX - 1)], 1u);
  }
  __syncthreads();
  hist[(int64_t)threadIdx.x * nblocks + blockIdx.x] = cnt[threadIdx.x];
}

__global__ void __launch_bounds__(SORT_THREADS) k_radix_scatter(const uint32_t* __restrict__ keys,
                                                                const uint32_t* __restrict__ vals, int64_t n,
                                                                int shift, const uint32_t* __restrict__ offs,
                                                                int nblocks, uint32_t* __restrict__ keys_out,
                                                                uint32_t* __restrict__ vals_out) {
  __shared__ uint32_t wcnt[SORT_WARPS][RADIX];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < SORT_WARPS * RADIX; i += SORT_THREADS) (&wcnt[0][0])[i] = 0;
  __syncthreads();
  // warp w owns [base + w*512, base + (w+1)*512), item-major then lane
  int64_t wbase = (int64_t)blockIdx.x * SORT_TILE + (int64_t)warp * (SORT_ITEMS * 32);
  uint32_t k[SORT_ITEMS], v[SORT_ITEMS], rank[SORT_ITEMS];
  unsigned lt = (1u << lane) - 1u;
#pragma unroll
  for (int it = 0; it < SORT_ITEMS; it++) {
    int64_t idx = wbase + it * 32 + lane;
    bool ok = idx < n;
    k[it] = ok ? keys[idx] : 0u;
    v[it] = ok ? vals[idx] : 0u;
    uint32_t d = (k[it] >> shift) & (RADIX - 1);
    uint32_t tag = ok ? d : (0x100u | (uint32_t)lane);
    unsigned peers = __match_any_sync(0xffffffffu, tag);
    int leader = __ffs(peers) - 1;
    uint32_t before = 0;
    if (ok && lane == leader) {
      before = wcnt[warp][d];
      wcnt[warp][d] = before + __popc(peers);
    }
    before = __shfl_sync(0xffffffffu, before, leader);
    rank[it] = before + __popc(peers & lt);
    __syncwarp();
  }
  __syncthreads();
  // exclusive scan over warps, per digit (thread t owns digit t)
  {
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < SORT_WARPS; w++) {
      uint32_t c = wcnt[w][threadIdx.x];
      wcnt[w][threadIdx.x] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int it = 0; it < SORT_ITEMS; it++) {
    int64_t idx = wbase + it * 32 + lane;
    if (idx >= n) continue;
    uint32_t d = (k[it] >> shift) & (RADIX - 1);
    uint32_t pos = offs[(int64_t)d * nblocks + blockIdx.x] + wcnt[warp][d] + rank[it];
    keys_out[pos] = k[it];
    vals_out[pos] = v[it];
  }
}

int scan_levels_size(int64_t n) {
  int64_t s = 16;
  while (n > 1) {
    n = (n + SCAN_TILE - 1) / SCAN_TILE;
    s += n + 16;
  }
  return (int)s;
}

// Recursive scan; `tmp` has room for all levels; the grand total goes to *total.
int scan_rec(emsesg_ctx* ctx, uint32_t* data, int64_t n, uint32_t* tmp, uint32_t* total) {
  int64_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
  uint32_t* part = tmp;
  EMSESG_LAUNCH(ctx, "scan_tile", k_scan_tile, (unsigned)nb, SCAN_THREADS, 0, data, n, part);
  if (nb == 1) {
    EMSESG_LAUNCH(ctx, "scan_total", k_copy_u32, 1, 1, 0, total, part);
    return EMSESG_OK;
  }
  int rc = scan_rec(ctx, part, nb, tmp + nb + 16, total);
  if (rc) return rc;
  EMSESG_LAUNCH(ctx, "scan_add", k_scan_add, (unsigned)((n + 255) / 256), 256, 0, data, n, part);
  return EMSESG_OK;
}

int ensure_scan_tmp(emsesg_ctx* ctx, int64_t n) {
  int64_t need = scan_levels_size(std::max<int64_t>(n, 2)) + 16;
  if (ctx->sort.scan_tmp_cap >= need) return EMSESG_OK;
  cudaStreamSynchronize(ctx->stream);
  cudaFree(ctx->sort.scan_tmp);
  ctx->sort.scan_tmp = nullptr;
  ctx->sort.scan_tmp_cap = 0;
  EMSESG_CUDA(ctx, cudaMalloc(&ctx->sort.scan_tmp, need * sizeof(uint32_t)));
  ctx->sort.scan_tmp_cap = need;
  return EMSESG_OK;
}

}  // namespace

// Exclusive scan in place; the total is left in ctx->sort.scan_tmp[0].
int exclusive_scan_u32(emsesg_ctx* ctx, uint32_t* data, int64_t n) {
  if (n <= 0) {
    int rc = ensure_scan_tmp(ctx, 2);
    if (rc) return rc;
    EMSESG_CUDA(ctx, cudaMemsetAsync(ctx->sort.scan_tmp, 0, sizeof(uint32_t), ctx->stream));
    return EMSESG_OK;
  }
  int rc = ensure_scan_tmp(ctx, n);
  if (rc) return rc;
  return scan_rec(ctx, data, n, ctx->sort.scan_tmp + 16, ctx->sort.scan_tmp);
}

int ensure_sort_scratch(emsesg_ctx* ctx, int64_t n) {
  n = std::max<int64_t>(n, 1);
  SortScratch& s = ctx->sort;
  if (s.cap < n) {
    cudaStreamSynchronize(ctx->stream);
    for (int b = 0; b < 2; b++) {
      cudaFree(s.keys[b]);
      cudaFree(s.vals[b]);
      s.keys[b] = s.vals[b] = nullptr;
    }
    s.cap = 0;
    for (int b = 0; b < 2; b++) {
      EMSESG_CUDA(ctx, cudaMalloc(&s.keys[b], n * sizeof(uint32_t)));
      EMSESG_CUDA(ctx, cudaMalloc(&s.vals[b], n * sizeof(uint32_t)));
    }
    s.cap = n;
  }
  int64_t nb = (n + SORT_TILE - 1) / SORT_TILE;
  int64_t hneed = nb * RADIX;
  if (s.hist_cap < hneed) {
    cudaStreamSynchronize(ctx->stream);
    cudaFree(s.hist);
    s.hist = nullptr;
    s.hist_cap = 0;
    EMSESG_CUDA(ctx, cudaMalloc(&s.hist, hneed * sizeof(uint32_t)));
    s.hist_cap = hneed;
  }
  return ensure_scan_tmp(ctx, std::max(hneed, n));
}

// Stable sort of (keys, vals) by the low key_bits bits of the keys.  The
// inputs are overwritten; *keys_out / *vals_out point at the sorted arrays
// (either the inputs or the other sort buffers).
int sort_pairs(emsesg_ctx* ctx, uint32_t* keys, uint32_t* vals, int64_t n, int key_bits, uint32_t** keys_out,
               uint32_t** vals_out) {
  int rc = ensure_sort_scratch(ctx, n);
  if (rc) return rc;
  uint32_t* kin = keys;
  uint32_t* vin = vals;
  uint32_t* kalt = (keys == ctx->sort.keys[0]) ? ctx->sort.keys[1] : ctx->sort.keys[0];
  uint32_t* valt = (vals == ctx->sort.vals[0]) ? ctx->sort.vals[1] : ctx->sort.vals[0];
  int nblocks = (int)((n + SORT_TILE - 1) / SORT_TILE);
  int passes = (key_bits + 7) / 8;
  for (int p = 0; p < passes; p++) {
    int shift = 8 * p;
    EMSESG_LAUNCH(ctx, "radix_hist", k_radix_hist, nblocks, SORT_THREADS, 0, kin, n, shift, ctx->sort.hist, nblocks);
    if ((rc = exclusive_scan_u32(ctx, ctx->sort.hist, (int64_t)nblocks * RADIX))) return rc;
    EMSESG_LAUNCH(ctx, "radix_scatter", k_radix_scatter, nblocks, SORT_THREADS, 0, kin, vin, n, shift,
                  ctx->sort.hist, nblocks, kalt, valt);
    std::swap(kin, kalt);
    std::swap(vin, valt);
  }
  *keys_out = kin;
  *vals_out = vin;
  return EMSESG_OK;
}

}  // namespace emsesg
