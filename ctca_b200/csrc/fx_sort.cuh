// fx_sort.cuh -- the tile-local counting sort of the FP32 form (included by
// fx.cu inside its private namespace, after fx_push.cuh).
//
// Between two sorts a particle moves by a fraction of a cell per step, so
// every particle of source tile t (its region of the last sort) lies in the
// "sort box" of t: the tile's cells plus one cell on every side (wrapped on
// the species' periodic axes).  The re-sort is then a counting sort whose
// buckets are cells, organised per source tile:
//
//   count   per (source tile, warp, box cell) counts of the live particles;
//   celltot per destination cell: the sum over the (at most 27) source tiles
//           whose box holds the cell; per destination tile: its total;
//   tiles   exclusive scan of the tile totals -> tile_start, tile_pad;
//   bases   per destination cell: its first rank (tile_start + scan over the
//           tile's cells), handed out to the source tiles in increasing tile
//           index: base[t'][bc'] = first rank of the cell's particles that
//           come from tile t'; empty slots of the new regions get DEAD;
//   rank    per source tile: each particle's rank = base[t][bc] + the counts
//           of the same cell in the tile's lower warps + its rank inside its
//           warp (rows in order, lanes in order, __match_any_sync) gives its
//           slot in the thread-major region of its new tile: inv[slot] = old
//           slot (4-byte scattered writes);
//   move    per destination tile, in groups of 32 columns or of the whole row: a window
//           of the tile's old region and the group's inv are staged in
//           shared memory (cp.async, double-buffered) and every slot takes
//           its particle from the window or, for particles from other tiles
//           or columns, from global memory (coalesced writes).
//
// Injected particles waiting in the tail zone join the same sort: the tail
// alone is radix-sorted by the tile-major cell key (a few million keys), its
// particles are added to the per-cell totals, and they take the last ranks
// of their cell, in the tail's sorted order (cell range end - (upper bound
// of the key - index)); the move then fetches them like particles of
// another tile.
//
// The order of equal-cell particles is thus (source tile, warp, row, lane):
// fixed by the data, so the sort is deterministic, and a particle is read
// twice (16 bytes to count and rank, 28 to move) and written once (28
// bytes), plus 4-byte slot indices.  Dead particles and empty slots are
// dropped (the compaction).  A particle outside its tile's sort box sets the
// stray flag; the host then sorts with the radix path instead.

struct LcsGeo {
  int n[3];      // grid cells
  int t[3];      // tile edge
  int nt[3];     // tiles per axis
  int bc[3];     // sort-box edge = t + 2
  int nbc;       // box cells
  int tcells;    // t[0]*t[1]*t[2]
  bool wrap[3];  // periodic particle axis (npbnd == 0)
};

// Block size of the per-cell kernels (one thread per cell of a tile of at
// most 8x8x8 cells).
constexpr int CELL_THREADS = 512;

__device__ __forceinline__ int lcs_axis(const LcsGeo& G, int d, int tile, int i) {
  int l = i - (tile * G.t[d] - 1);
  if (G.wrap[d]) {
    if (l < 0) l += G.n[d];
    else if (l >= G.n[d]) l -= G.n[d];
  }
  return (l >= 0 && l < G.bc[d]) ? l : -1;
}

// Box cell of cell (i,j,k) in the sort box of tile (tx,ty,tz), or -1.
__device__ __forceinline__ int lcs_box_cell(const LcsGeo& G, int tx, int ty, int tz, int i, int j, int k) {
  int a = lcs_axis(G, 0, tx, i), b = lcs_axis(G, 1, ty, j), c = lcs_axis(G, 2, tz, k);
  if (a < 0 || b < 0 || c < 0) return -1;
  return a + G.bc[0] * (b + G.bc[1] * c);
}

// Tiles along one axis whose sort box holds cell index i, ascending,
// without repeats (the tile of i, and a neighbour when i lies in its guard).
__device__ __forceinline__ int lcs_cand(const LcsGeo& G, int d, int i, int (&out)[3]) {
  const int c = i / G.t[d];
  int m = 0;
  int v[3] = {c - 1, c, c + 1};
  int w[3];
  for (int q = 0; q < 3; q++) {
    int x = v[q];
    if (x < 0 || x >= G.nt[d]) {
      if (!G.wrap[d]) continue;
      x = (x + G.nt[d]) % G.nt[d];
    }
    if (lcs_axis(G, d, x, i) < 0) continue;
    w[m++] = x;
  }
  // sort the (at most 3) entries and drop repeats
  for (int a = 1; a < m; a++)
    for (int b = a; b > 0 && w[b - 1] > w[b]; b--) { int s = w[b]; w[b] = w[b - 1]; w[b - 1] = s; }
  int k = 0;
  for (int a = 0; a < m; a++)
    if (k == 0 || out[k - 1] != w[a]) out[k++] = w[a];
  return k;
}

__device__ __forceinline__ void tile_xyz(const Geo& g, int64_t t, int& tx, int& ty, int& tz) {
  tx = (int)(t % g.nt[0]);
  ty = (int)((t / g.nt[0]) % g.nt[1]);
  tz = (int)(t / ((int64_t)g.nt[0] * g.nt[1]));
}

// count: per (source tile, warp, box cell).  grid = ntiles, block = PUSH_THREADS.
__global__ void __launch_bounds__(PUSH_THREADS) k_lcs_count(const float4* __restrict__ pos,
                                                            const int64_t* __restrict__ ts,
                                                            const int64_t* __restrict__ tp, Geo g, LcsGeo G,
                                                            uint32_t* __restrict__ wcnt, uint32_t* __restrict__ cnt,
                                                            int* stray) {
  extern __shared__ uint32_t hist[];  // [PUSH_WARPS][nbc]
  const int t = blockIdx.x, tid = threadIdx.x, warp = tid >> 5;
  for (int e = tid; e < PUSH_WARPS * G.nbc; e += PUSH_THREADS) hist[e] = 0;
  __syncthreads();
  int tx, ty, tz;
  tile_xyz(g, t, tx, ty, tz);
  const int64_t n = ts[t + 1] - ts[t];
  const int L = (int)((n + PUSH_THREADS - 1) / PUSH_THREADS);
  bool bad = false;
  const float4* src = pos + tp[t];
#pragma unroll 4
  for (int r = 0; r < L; r++) {
    const uint32_t cell = (uint32_t)__float_as_int(src[r * PUSH_THREADS + tid].w);
    if (cell == DEAD) continue;
    int i, j, k;
    unpack(g, cell, i, j, k);
    const int bc = lcs_box_cell(G, tx, ty, tz, i, j, k);
    if (bc < 0) { bad = true; continue; }
    atomicAdd(&hist[warp * G.nbc + bc], 1u);
  }
  __syncthreads();
  uint32_t* wc = wcnt + (int64_t)t * PUSH_WARPS * G.nbc;
  uint32_t* c = cnt + (int64_t)t * G.nbc;
  for (int b = tid; b < G.nbc; b += PUSH_THREADS) {
    uint32_t sum = 0;
    for (int w = 0; w < PUSH_WARPS; w++) {
      uint32_t h = hist[w * G.nbc + b];
      wc[w * G.nbc + b] = h;
      sum += h;
    }
    c[b] = sum;
  }
  if (bad) atomicOr(stray, 1);
}

// celltot: per destination cell, the sum over the source tiles holding it;
// per destination tile its total.  grid = ntiles, block = CELL_THREADS (>= tcells).
__global__ void __launch_bounds__(CELL_THREADS) k_lcs_celltot(const uint32_t* __restrict__ cnt, Geo g, LcsGeo G,
                                                              uint32_t* __restrict__ celltot,
                                                              int64_t* __restrict__ tiletot, const int* stray) {
  __shared__ uint32_t part[CELL_THREADS / 32];
  if (*stray) return;  // a particle left its sort box: this sort is skipped (see fx_local_sort)
  const int t = blockIdx.x, tid = threadIdx.x;
  int tx, ty, tz;
  tile_xyz(g, t, tx, ty, tz);
  uint32_t tot = 0;
  if (tid < G.tcells) {
    const int i = tx * G.t[0] + tid % G.t[0];
    const int j = ty * G.t[1] + (tid / G.t[0]) % G.t[1];
    const int k = tz * G.t[2] + tid / (G.t[0] * G.t[1]);
    if (i < G.n[0] && j < G.n[1] && k < G.n[2]) {
      int cx[3], cy[3], cz[3];
      const int mx = lcs_cand(G, 0, i, cx), my = lcs_cand(G, 1, j, cy), mz = lcs_cand(G, 2, k, cz);
      for (int c = 0; c < mz; c++)
        for (int b = 0; b < my; b++)
          for (int a = 0; a < mx; a++) {
            const int bc = lcs_box_cell(G, cx[a], cy[b], cz[c], i, j, k);
            if (bc < 0) continue;
            const int64_t tt = cx[a] + (int64_t)g.nt[0] * (cy[b] + (int64_t)g.nt[1] * cz[c]);
            tot += cnt[tt * G.nbc + bc];
          }
    }
    celltot[(int64_t)t * G.tcells + tid] = tot;
  }
  // block sum
  uint32_t v = tot;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((tid & 31) == 0) part[tid >> 5] = v;
  __syncthreads();
  if (tid == 0) {
    int64_t s = 0;
    for (int w = 0; w < CELL_THREADS / 32; w++) s += part[w];
    tiletot[t] = s;
  }
}

// tiles: exclusive scan of the tile totals (one block of 1024 threads):
// tile_start, tile_pad (whole rows per tile), live count and slot count.
__global__ void __launch_bounds__(1024) k_lcs_tiles(const int64_t* __restrict__ tiletot, int64_t ntiles,
                                                    int64_t* ts, int64_t* tp, int64_t* count, int64_t* slots,
                                                    const int* stray) {
  __shared__ int64_t pa[1024], pb[1024];
  if (*stray) return;
  const int tid = threadIdx.x;
  const int64_t per = (ntiles + 1023) / 1024;
  const int64_t t0 = tid * per, t1 = min(ntiles, t0 + per);
  int64_t sa = 0, sb = 0;
  for (int64_t t = t0; t < t1; t++) {
    sa += tiletot[t];
    sb += (tiletot[t] + PUSH_THREADS - 1) / PUSH_THREADS * PUSH_THREADS;
  }
  pa[tid] = sa;
  pb[tid] = sb;
  __syncthreads();
  for (int d = 1; d < 1024; d <<= 1) {
    int64_t va = tid >= d ? pa[tid - d] : 0, vb = tid >= d ? pb[tid - d] : 0;
    __syncthreads();
    pa[tid] += va;
    pb[tid] += vb;
    __syncthreads();
  }
  int64_t ra = pa[tid] - sa, rb = pb[tid] - sb;
  for (int64_t t = t0; t < t1; t++) {
    ts[t] = ra;
    tp[t] = rb;
    ra += tiletot[t];
    rb += (tiletot[t] + PUSH_THREADS - 1) / PUSH_THREADS * PUSH_THREADS;
  }
  if (tid == 1023) {
    ts[ntiles] = pa[1023];
    tp[ntiles] = pb[1023];
    *count = pa[1023];
    *slots = pb[1023];
  }
}

// bases: first rank of every (source tile, box cell); DEAD in the empty
// slots of the new region.  grid = ntiles (destination tiles), block = CELL_THREADS.
__global__ void __launch_bounds__(CELL_THREADS) k_lcs_bases(const uint32_t* __restrict__ cnt,
                                                            uint32_t* celltot, Geo g, LcsGeo G,
                                                            const int64_t* __restrict__ ts,
                                                            const int64_t* __restrict__ tp, uint32_t* __restrict__ base,
                                                            uint32_t* __restrict__ inv, const int* stray) {
  __shared__ uint32_t sc[CELL_THREADS];
  if (*stray) return;
  const int t = blockIdx.x, tid = threadIdx.x;
  int tx, ty, tz;
  tile_xyz(g, t, tx, ty, tz);
  const uint32_t mine = tid < G.tcells ? celltot[(int64_t)t * G.tcells + tid] : 0u;
  // exclusive scan over the tile's cells (cell order = the sort key order)
  sc[tid] = mine;
  __syncthreads();
  for (int d = 1; d < CELL_THREADS; d <<= 1) {
    uint32_t v = tid >= d ? sc[tid - d] : 0u;
    __syncthreads();
    sc[tid] += v;
    __syncthreads();
  }
  if (tid < G.tcells) {
    const int i = tx * G.t[0] + tid % G.t[0];
    const int j = ty * G.t[1] + (tid / G.t[0]) % G.t[1];
    const int k = tz * G.t[2] + tid / (G.t[0] * G.t[1]);
    if (i < G.n[0] && j < G.n[1] && k < G.n[2]) {
      uint32_t run = (uint32_t)ts[t] + sc[tid] - mine;
      int cx[3], cy[3], cz[3];
      const int mx = lcs_cand(G, 0, i, cx), my = lcs_cand(G, 1, j, cy), mz = lcs_cand(G, 2, k, cz);
      for (int c = 0; c < mz; c++)
        for (int b = 0; b < my; b++)
          for (int a = 0; a < mx; a++) {
            const int bc = lcs_box_cell(G, cx[a], cy[b], cz[c], i, j, k);
            if (bc < 0) continue;
            const int64_t tt = cx[a] + (int64_t)g.nt[0] * (cy[b] + (int64_t)g.nt[1] * cz[c]);
            base[tt * G.nbc + bc] = run;
            run += cnt[tt * G.nbc + bc];
          }
    }
    // the cell's end rank (its tail particles take the ranks before it)
    celltot[(int64_t)t * G.tcells + tid] = (uint32_t)ts[t] + sc[tid];
  }
  // empty slots of the new region
  const int64_t n = ts[t + 1] - ts[t];
  if (n > 0) {
    const int L = (int)((n + PUSH_THREADS - 1) / PUSH_THREADS);
    for (int64_t q = n + tid; q < (int64_t)L * PUSH_THREADS; q += CELL_THREADS) {
      const int64_t slot = tp[t] + (q % L) * PUSH_THREADS + q / L;
      inv[slot] = DEAD;
    }
  }
}

// q / d for 32-bit q and d >= 1 by one 64-bit high multiply with
// M = ceil(2^64 / d) (Lemire, Kaser and Kurz, "Faster remainder by direct
// computation", 2019); d = 1 is passed through.
__host__ __device__ __forceinline__ uint64_t fastdiv_mul(uint32_t d) {
  return d > 1 ? ~0ull / d + 1 : 0ull;
}
__device__ __forceinline__ uint32_t fastdiv(uint32_t q, uint32_t d, uint64_t M) {
  return d > 1 ? (uint32_t)__umul64hi(M, (uint64_t)q) : q;
}

// rank: every live particle of source tile t gets its slot in the new
// regions; inv[new slot] = old slot (4-byte scattered writes).  grid =
// ntiles, block = PUSH_THREADS, shared = PUSH_WARPS * nbc * 4.

__global__ void __launch_bounds__(PUSH_THREADS) k_lcs_rank(const float4* __restrict__ pos,
                                                              const int64_t* __restrict__ ts,
                                                              const int64_t* __restrict__ tp, Geo g, LcsGeo G,
                                                              const uint32_t* __restrict__ wcnt,
                                                              const uint32_t* __restrict__ base,
                                                              const int64_t* __restrict__ ts2,
                                                              const int64_t* __restrict__ tp2,
                                                              uint32_t* __restrict__ inv, int* status,
                                                              long long* diag, const int* stray) {
  extern __shared__ uint32_t wb[];  // [PUSH_WARPS][nbc] next rank of (warp, box cell)
  if (*stray) return;
  const int t = blockIdx.x, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const unsigned lt = (1u << lane) - 1u;
  const uint32_t* wc = wcnt + (int64_t)t * PUSH_WARPS * G.nbc;
  for (int b = tid; b < G.nbc; b += PUSH_THREADS) {
    uint32_t run = base[(int64_t)t * G.nbc + b];
    for (int w = 0; w < PUSH_WARPS; w++) {
      wb[w * G.nbc + b] = run;
      run += wc[w * G.nbc + b];
    }
  }
  int tx, ty, tz;
  tile_xyz(g, t, tx, ty, tz);
  // the 27 tiles around this one (the destinations of its particles): first
  // rank, count, rows with their division multiplier, region start; a
  // sort-box cell's side on each axis (below, inside, above the tile) picks
  // the entry
  __shared__ uint32_t nq0[27], nnd[27], nld[27];
  __shared__ uint64_t nmul[27];
  __shared__ int64_t ntp[27];
  if (tid < 27) {
    const int d3[3] = {tid % 3 - 1, (tid / 3) % 3 - 1, tid / 9 - 1};
    const int c3[3] = {tx, ty, tz};
    bool ok = true;
    int64_t td = 0, mul = 1;
    for (int d = 0; d < 3; d++) {
      int x = c3[d] + d3[d];
      if (x < 0 || x >= g.nt[d]) {
        if (G.wrap[d]) x = (x + g.nt[d]) % g.nt[d];
        else ok = false;
      }
      td += mul * x;
      mul *= g.nt[d];
    }
    const int64_t nd = ok ? ts2[td + 1] - ts2[td] : 0;
    nq0[tid] = ok ? (uint32_t)ts2[td] : 0u;
    nnd[tid] = (uint32_t)nd;
    const uint32_t ld = (uint32_t)((nd + PUSH_THREADS - 1) / PUSH_THREADS);
    nld[tid] = ld;
    nmul[tid] = fastdiv_mul(ld);
    ntp[tid] = ok ? tp2[td] : 0;
  }
  __syncthreads();
  const int64_t n = ts[t + 1] - ts[t];
  const int L = (int)((n + PUSH_THREADS - 1) / PUSH_THREADS);
  const int64_t s0 = tp[t];
  uint32_t* mywb = wb + warp * G.nbc;
  // the tile's own cells per axis (the last tile of an axis whose length is
  // not a multiple of the tile is shorter; on a periodic axis its sort box
  // then reaches past the grid's end onto the next tile's cells): box
  // position 0 is the tile below, 1..ext its own cells, beyond them the tile
  // above
  const int ext0 = min(G.t[0], G.n[0] - tx * G.t[0]), ext1 = min(G.t[1], G.n[1] - ty * G.t[1]),
            ext2 = min(G.t[2], G.n[2] - tz * G.t[2]);
  // the cells of the next rows are loaded ahead
  constexpr int AHEAD = 4;
  uint32_t cr[AHEAD];
#pragma unroll
  for (int q = 0; q < AHEAD; q++)
    cr[q] = q < L ? (uint32_t)__float_as_int(pos[s0 + (int64_t)q * PUSH_THREADS + tid].w) : DEAD;
  for (int r = 0; r < L; r++) {
    const int64_t m = s0 + (int64_t)r * PUSH_THREADS + tid;
    const uint32_t cell = cr[0];
#pragma unroll
    for (int q = 0; q < AHEAD - 1; q++) cr[q] = cr[q + 1];
    cr[AHEAD - 1] = r + AHEAD < L ? (uint32_t)__float_as_int(pos[m + (int64_t)AHEAD * PUSH_THREADS].w) : DEAD;
    int bc = -1, nb = 0;
    if (cell != DEAD) {
      int i, j, k;
      unpack(g, cell, i, j, k);
      const int a = lcs_axis(G, 0, tx, i), b = lcs_axis(G, 1, ty, j), c = lcs_axis(G, 2, tz, k);
      if ((a | b | c) >= 0) {  // else a stray: the radix path sorts
        bc = a + G.bc[0] * (b + G.bc[1] * c);
        nb = (a == 0 ? 0 : (a <= ext0 ? 1 : 2)) + 3 * (b == 0 ? 0 : (b <= ext1 ? 1 : 2)) +
             9 * (c == 0 ? 0 : (c <= ext2 ? 1 : 2));
      }
    }
    const unsigned peers = __match_any_sync(0xffffffffu, bc);
    const uint32_t rank = bc >= 0 ? mywb[bc] + __popc(peers & lt) : 0u;
    __syncwarp();
    if (bc >= 0 && (peers & lt) == 0) mywb[bc] += __popc(peers);
    __syncwarp();
    if (bc < 0) continue;
    // the destination tile's thread-major slot
    const uint32_t q = rank - nq0[nb];
    if (q >= nnd[nb]) {
      report_bad(status, diag, SITE_FX_SORT, m, (long long)cell);
      continue;
    }
    const uint32_t Ld = nld[nb];
    const uint32_t col = fastdiv(q, Ld, nmul[nb]);
    inv[ntp[nb] + (q - col * Ld) * PUSH_THREADS + col] = (uint32_t)m;
  }
}

// move: the new region of destination tile t, in groups of GW columns.  A
// particle that stayed in its tile keeps about its column (its rank moves by
// the net count change of the cells before it), so each group takes its
// particles from a window of GW + 8 source columns (all rows of the tile's
// old region), centred on the old column of the group's middle slot, or,
// when one came from elsewhere, from global memory; the writes go row by row
// (coalesced).  The window and the group's columns of inv are staged in
// shared memory with cp.async, double-buffered: group g+1's copies are in
// flight while group g is written.  The group width is the widest of 32,
// 96, 160 columns and the whole row (those that divide the row) whose group
// fits the staged slots at the tile's row count, so that a tile of few rows
// is moved in few groups.
//
// Two shapes (MoveBig, MoveSmall), picked per sort by the mean rows per
// tile: tiles of many rows need big windows (80 rows: 200 KB of shared
// memory, copies that skip L1); for tiles of at most 40 rows the buffers
// take half that, and the copies go through L1, which then holds the
// recent columns of the old region: the particles that changed cell along
// z (whose rank moves by a z-layer, tens of columns) are found there.
// A third shape (MoveMid) for tiles of up to 56 rows keeps two groups'
// copies in flight (three buffers) while one group is written.
// grid = ntiles, block = PUSH_THREADS (one CTA per SM), shared =
// Cfg::NBUF * Cfg::BUF.
template <int WIN_, int SLOTS_, bool CA_, int NBUF_ = 2>
struct MoveCfg {
  static constexpr int WIN = WIN_;      // window particles of one buffer
  static constexpr int SLOTS = SLOTS_;  // slots of one group (staged inv)
  static constexpr bool CA = CA_;       // copies cached in L1
  static constexpr int NBUF = NBUF_;    // buffers: NBUF - 1 groups in flight while one is written
  static constexpr int K = (SLOTS + PUSH_THREADS - 1) / PUSH_THREADS;  // slots of a thread per group
  static constexpr int BUF = WIN * (16 + 3 * 4) + SLOTS * 4;          // bytes of one buffer
  static_assert(NBUF == 2 || NBUF == 3, "double or triple buffering");
};
using MoveBig = MoveCfg<3200, 2560, false>;      // up to 80 rows of 40 columns
using MoveMid = MoveCfg<2240, 1792, false, 3>;   // up to 56 rows of 40 columns, two groups in flight
using MoveSmall = MoveCfg<1600, 1280, true>;     // up to 40 rows of 40 columns
constexpr int MOVE_SMALL_ROWS = 32;              // mean rows per tile up to which MoveSmall is used
constexpr int MOVE_MID_ROWS = 48;                // then MoveMid up to this mean
constexpr int MOVE_MAXGROUPS = PUSH_THREADS / 32;
template <class Cfg>
inline int move_smem() { return Cfg::NBUF * Cfg::BUF; }
static_assert(PUSH_THREADS % 32 == 0, "32-column groups divide the row");

template <bool CA>
__device__ __forceinline__ void cpa16(void* dst, const void* src) {
  if (CA)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(dst)), "l"(src) : "memory");
  else
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpa_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
__device__ __forceinline__ bool al16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

// One destination tile with groups of GW columns (see k_lcs_move).
template <class Cfg, int GW>
__device__ __forceinline__ void move_tile(const float4* __restrict__ pos, const float* __restrict__ vx,
                                          const float* __restrict__ vy, const float* __restrict__ vz,
                                          const uint32_t* __restrict__ inv, float4* __restrict__ pos2,
                                          float* __restrict__ vx2, float* __restrict__ vy2, float* __restrict__ vz2,
                                          int Ld, int Ls, int64_t sbase, int64_t d0, bool any_src, float4* msm,
                                          int* wlo) {
  constexpr int WC = GW + 8 < PUSH_THREADS ? GW + 8 : PUSH_THREADS;  // window columns, a multiple of 4
  constexpr int NG = PUSH_THREADS / GW;
  constexpr int VCH = WC / 4;  // 16-byte chunks of a velocity row
  constexpr int GCH = GW / 4;  // 16-byte chunks of a group's inv row
  static_assert(PUSH_THREADS % GW == 0 && WC % 4 == 0 && GW % 32 == 0, "group shape");
  const int tid = threadIdx.x;
  const int64_t send = sbase + (int64_t)Ls * PUSH_THREADS;
  constexpr int MOVE_WIN = Cfg::WIN, MOVE_K = Cfg::K, MOVE_BUF = Cfg::BUF;
  const bool win = any_src && Ls * WC <= MOVE_WIN && al16(pos + sbase) && al16(vx + sbase) && al16(vy + sbase) &&
                   al16(vz + sbase);
  const bool sinv = Ld * GW <= Cfg::SLOTS && al16(inv + d0);
  // the window of every group, from the old slot of the group's middle slot
  if (win && tid < NG) {
    const int c0 = tid * GW;
    const uint32_t s = inv[d0 + (int64_t)(Ld / 2) * PUSH_THREADS + c0 + GW / 2];
    int col = c0 + GW / 2;
    if (s != DEAD && (int64_t)s >= sbase && (int64_t)s < send) col = (int)(((int64_t)s - sbase) % PUSH_THREADS);
    wlo[tid] = min(max(col - WC / 2, 0), PUSH_THREADS - WC) & ~3;
  }
  __syncthreads();
  auto stage = [&](int grp) {
    char* buf = reinterpret_cast<char*>(msm) + (grp % Cfg::NBUF) * MOVE_BUF;
    float4* wpos = reinterpret_cast<float4*>(buf);
    float* wv = reinterpret_cast<float*>(wpos + MOVE_WIN);
    uint32_t* winv = reinterpret_cast<uint32_t*>(wv + 3 * MOVE_WIN);
    if (win) {
      const int lo = wlo[grp];
      const float4* ps = pos + sbase + lo;
      for (int e = tid; e < Ls * WC; e += PUSH_THREADS) {
        const int row = e / WC, col = e - row * WC;
        cpa16<Cfg::CA>(wpos + e, ps + row * PUSH_THREADS + col);
      }
      const float* v3[3] = {vx + sbase + lo, vy + sbase + lo, vz + sbase + lo};
#pragma unroll
      for (int arr = 0; arr < 3; arr++)
        for (int h = tid; h < Ls * VCH; h += PUSH_THREADS) {
          const int row = h / VCH, ch = h - row * VCH;
          cpa16<Cfg::CA>(wv + arr * MOVE_WIN + row * WC + 4 * ch, v3[arr] + row * PUSH_THREADS + 4 * ch);
        }
    }
    if (sinv) {
      const uint32_t* is = inv + d0 + grp * GW;
      for (int e = tid; e < Ld * GCH; e += PUSH_THREADS) {
        const int row = e / GCH, ch = e - row * GCH;
        cpa16<Cfg::CA>(winv + row * GW + 4 * ch, is + row * PUSH_THREADS + 4 * ch);
      }
    }
    cpa_commit();
  };
  stage(0);
  if (Cfg::NBUF == 3 && NG > 1) stage(1);
  for (int grp = 0; grp < NG; grp++) {
    if (Cfg::NBUF == 3) {
      if (grp + 2 < NG) {
        stage(grp + 2);
        cpa_wait<2>();
      } else if (grp + 1 < NG) {
        cpa_wait<1>();
      } else {
        cpa_wait<0>();
      }
    } else if (grp + 1 < NG) {
      stage(grp + 1);
      cpa_wait<1>();
    } else {
      cpa_wait<0>();
    }
    __syncthreads();
    const char* buf = reinterpret_cast<const char*>(msm) + (grp % Cfg::NBUF) * MOVE_BUF;
    const float4* wpos = reinterpret_cast<const float4*>(buf);
    const float* wvx = reinterpret_cast<const float*>(wpos + MOVE_WIN);
    const float* wvy = wvx + MOVE_WIN;
    const float* wvz = wvy + MOVE_WIN;
    const uint32_t* winv = reinterpret_cast<const uint32_t*>(wvz + MOVE_WIN);
    const int64_t g0 = d0 + grp * GW;
    const int lo = win ? wlo[grp] : 0;
    // MOVE_K slots of a thread at a time (all of the group's when its inv is
    // staged): every load is issued before the first store, so the
    // particles gathered from global memory are in flight together
    for (int e0 = 0; e0 < Ld * GW; e0 += MOVE_K * PUSH_THREADS) {
      float4 p[MOVE_K];
      float a[MOVE_K], b[MOVE_K], c[MOVE_K];
#pragma unroll
      for (int k = 0; k < MOVE_K; k++) {
        const int e = e0 + tid + k * PUSH_THREADS;
        p[k] = make_float4(0.f, 0.f, 0.f, __int_as_float((int)DEAD));
        a[k] = b[k] = c[k] = 0.f;
        if (e < Ld * GW) {
          const int row = e / GW;
          const uint32_t src = sinv ? winv[e] : inv[g0 + (int64_t)row * PUSH_THREADS + (e - row * GW)];
          if (src != DEAD) {
            // 32-bit offset into the old region (regions hold fewer than 2^31 slots)
            const uint32_t rel = src - (uint32_t)sbase;
            const int cc = win && rel < (uint32_t)(send - sbase) ? (int)(rel % PUSH_THREADS) - lo : -1;
            if (cc >= 0 && cc < WC) {
              const int w = (int)(rel / PUSH_THREADS) * WC + cc;
              p[k] = wpos[w];
              a[k] = wvx[w];
              b[k] = wvy[w];
              c[k] = wvz[w];
            } else {
              p[k] = pos[src];
              a[k] = vx[src];
              b[k] = vy[src];
              c[k] = vz[src];
            }
          }
        }
      }
#pragma unroll
      for (int k = 0; k < MOVE_K; k++) {
        const int e = e0 + tid + k * PUSH_THREADS;
        if (e < Ld * GW) {
          const int row = e / GW;
          const int64_t m = g0 + (int64_t)row * PUSH_THREADS + (e - row * GW);
          pos2[m] = p[k];
          vx2[m] = a[k];
          vy2[m] = b[k];
          vz2[m] = c[k];
        }
      }
    }
    __syncthreads();  // this buffer is staged again for group grp + NBUF
  }
}

template <class Cfg>
__global__ void __launch_bounds__(PUSH_THREADS, 1) k_lcs_move(const float4* __restrict__ pos,
                                                              const float* __restrict__ vx,
                                                              const float* __restrict__ vy,
                                                              const float* __restrict__ vz,
                                                              const int64_t* __restrict__ ts,
                                                              const int64_t* __restrict__ tp,
                                                              const int64_t* __restrict__ ts2,
                                                              const int64_t* __restrict__ tp2,
                                                              const uint32_t* __restrict__ inv, float4* __restrict__ pos2,
                                                              float* __restrict__ vx2, float* __restrict__ vy2,
                                                              float* __restrict__ vz2, const int* stray) {
  extern __shared__ float4 msm[];  // two buffers: window pos, vx, vy, vz, then the group's inv
  __shared__ int wlo[MOVE_MAXGROUPS];
  if (*stray) return;
  const int t = blockIdx.x;
  const int64_t nd = ts2[t + 1] - ts2[t];
  if (nd <= 0) return;
  const int Ld = (int)((nd + PUSH_THREADS - 1) / PUSH_THREADS);
  const int64_t ns = ts[t + 1] - ts[t];
  const int Ls = (int)((ns + PUSH_THREADS - 1) / PUSH_THREADS);
  const int R = max(Ls, Ld);
  if (R * PUSH_THREADS <= Cfg::SLOTS) {
    move_tile<Cfg, PUSH_THREADS>(pos, vx, vy, vz, inv, pos2, vx2, vy2, vz2, Ld, Ls, tp[t], tp2[t], ns > 0, msm, wlo);
    return;
  }
  if constexpr (PUSH_THREADS % 160 == 0) {
    if (R * 160 <= Cfg::SLOTS) {
      move_tile<Cfg, 160>(pos, vx, vy, vz, inv, pos2, vx2, vy2, vz2, Ld, Ls, tp[t], tp2[t], ns > 0, msm, wlo);
      return;
    }
  }
  if constexpr (PUSH_THREADS % 96 == 0) {
    if (R * 96 <= Cfg::SLOTS) {
      move_tile<Cfg, 96>(pos, vx, vy, vz, inv, pos2, vx2, vy2, vz2, Ld, Ls, tp[t], tp2[t], ns > 0, msm, wlo);
      return;
    }
  }
  move_tile<Cfg, 32>(pos, vx, vy, vz, inv, pos2, vx2, vy2, vz2, Ld, Ls, tp[t], tp2[t], ns > 0, msm, wlo);
}

// Inside a CUDA graph the host cannot switch to the radix sort when a
// particle has left its tile's sort box; the sort kernels above then return
// at once and this one keeps the current order instead: the new buffers get
// the old regions slot for slot (inv = identity).  The push handles a
// particle outside its tile's box on its general path (global gather and
// deposits), so the step stays correct, only slower, until the next sort
// outside a graph.  Does nothing when no particle strayed.
__global__ void __launch_bounds__(256) k_lcs_keep(const int* stray, const float4* __restrict__ pos,
                                                  const float* __restrict__ vx, const float* __restrict__ vy,
                                                  const float* __restrict__ vz, const int64_t* __restrict__ ts,
                                                  const int64_t* __restrict__ tp, int64_t ntiles, float4* pos2,
                                                  float* vx2, float* vy2, float* vz2, int64_t* ts2, int64_t* tp2,
                                                  uint32_t* inv) {
  if (!*stray) return;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (int64_t t = i0; t <= ntiles; t += stride) {
    ts2[t] = ts[t];
    tp2[t] = tp[t];
  }
  const int64_t n = tp[ntiles];
  for (int64_t i = i0; i < n; i += stride) {
    pos2[i] = pos[i];
    vx2[i] = vx[i];
    vy2[i] = vy[i];
    vz2[i] = vz[i];
    inv[i] = __float_as_uint(pos[i].w) == DEAD ? DEAD : (uint32_t)i;
  }
}

// The tail's particles in the per-cell and per-tile totals.  keys: the
// tail's sorted tile-major cell keys (deadkey for dead particles).
__global__ void __launch_bounds__(256) k_lcs_tail_count(const uint32_t* __restrict__ keys, int64_t nt,
                                                        uint32_t deadkey, int tcells, uint32_t* celltot,
                                                        unsigned long long* tiletot, const int* stray) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nt || *stray) return;
  const uint32_t key = keys[i];
  if (key >= deadkey) return;
  atomicAdd(&celltot[key], 1u);
  atomicAdd(&tiletot[key / (uint32_t)tcells], 1ull);
}

// The new slot of every live tail particle: the last ranks of its cell, in
// the tail's sorted order.  cellend: per (tile, cell) the end rank (from
// k_lcs_bases); inv[new slot] = old (tail) slot.
__global__ void __launch_bounds__(256) k_lcs_tail_inv(const uint32_t* __restrict__ keys,
                                                      const uint32_t* __restrict__ vals, int64_t nt, uint32_t deadkey,
                                                      int tcells, const uint32_t* __restrict__ cellend,
                                                      const int64_t* __restrict__ ts, const int64_t* __restrict__ tp,
                                                      uint32_t* inv, const int* stray) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nt || *stray) return;
  const uint32_t key = keys[i];
  if (key >= deadkey) return;
  // upper bound of the key in the sorted tail
  int64_t lo = i + 1, hi = nt;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (keys[mid] <= key) lo = mid + 1;
    else hi = mid;
  }
  const int64_t t = key / (uint32_t)tcells;
  const int64_t q = (int64_t)cellend[key] - (lo - i) - ts[t];  // rank inside the tile
  const int64_t n = ts[t + 1] - ts[t];
  const int64_t L = (n + PUSH_THREADS - 1) / PUSH_THREADS;
  inv[tp[t] + (q % L) * PUSH_THREADS + q / L] = vals[i];
}
