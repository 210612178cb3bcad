// fx.cu -- the FP32 / fixed-point form of the EMSES particle step.
//
// Particle state (per species region, 28 bytes a particle):
//   pos[m] = {ox, oy, oz, cell}: in-cell offsets in [0,1) (FP32) and the
//            packed cell index i | j<<bx | k<<(bx+by) (int32 bits; all ones
//            marks a dead particle),
//   vx[m], vy[m], vz[m]: FP32 velocities in internal units.
// Particles stay sorted by the tile-major cell key (8x8x8 cell tiles by
// default); tile_start[t] .. tile_start[t+1] is the slice of tile t at the
// last sort, and one CTA pushes one tile of one species.
//
// The step kernel fuses, per particle: the trilinear E/B gather from the
// FP32 node field (grdcrt output), the Buneman-Boris push, the move and the
// outer boundary rules of psolve1.F90:366-606 evaluated on (integer cell,
// FP32 offset) pairs, the zigzag current of psolve1.F90:717-789 and the CIC
// charge of charge.F90:59-80 at the new position (fx_push.cuh).  Deposits
// are summed per cell in registers along each thread's sorted slice,
// converted to int64 fixed point at 2^40 and added into a shared-memory
// accumulator covering the tile plus a 2-cell guard; the CTA then adds its
// accumulator into the global int64 arrays.  Integer adds commute, so the
// global sums do not depend on the order in which CTAs and atomics run, and
// the FP32 partial sums depend only on the sorted order and the fixed thread
// slicing, so every run gives the same bits.
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "slab.cuh"

namespace emsesg {

namespace {

constexpr uint32_t DEAD = 0xFFFFFFFFu;
constexpr double FIX_INV = 1.0 / 1099511627776.0;

struct Geo {
  int nx, ny, nz;
  int bx, by;        // packed cell bit widths (x, y)
  uint32_t mx, my;   // masks
  int t[3], nt[3];   // sort tile and tile counts
};

__device__ __forceinline__ void unpack(const Geo& g, uint32_t c, int& i, int& j, int& k) {
  i = (int)(c & g.mx);
  j = (int)((c >> g.bx) & g.my);
  k = (int)(c >> (g.bx + g.by));
}
__device__ __forceinline__ uint32_t pack(const Geo& g, int i, int j, int k) {
  return (uint32_t)i | ((uint32_t)j << g.bx) | ((uint32_t)k << (g.bx + g.by));
}

// ---------------------------------------------------------------- fields
// FP32 node field from the staggered FP64 eb (grdcrt.F90:156-169, 214-230),
// nodes 0..n on every axis.
__global__ void k_grdcrt32(const double* __restrict__ eb, float4* __restrict__ f0, float4* __restrict__ f1,
                           FieldDesc fe, int nx, int ny, int nz, double e0x, double e0y, double e0z, double b0x,
                           double b0y, double b0z) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t ex = nx + 1, ey = ny + 1, ez = nz + 1;
  if (t >= ex * ey * ez) return;
  int i = (int)(t % ex), j = (int)((t / ex) % ey), k = (int)(t / (ex * ey));
  double wex = 0.5 * (eb[fe.at(0, i, j, k)] + eb[fe.at(0, i - 1, j, k)]) + e0x;
  double wey = 0.5 * (eb[fe.at(1, i, j, k)] + eb[fe.at(1, i, j - 1, k)]) + e0y;
  double wez = 0.5 * (eb[fe.at(2, i, j, k)] + eb[fe.at(2, i, j, k - 1)]) + e0z;
  double wbx = 0.25 * (eb[fe.at(3, i, j, k)] + eb[fe.at(3, i, j - 1, k)] + eb[fe.at(3, i, j, k - 1)] +
                       eb[fe.at(3, i, j - 1, k - 1)]) + b0x;
  double wby = 0.25 * (eb[fe.at(4, i, j, k)] + eb[fe.at(4, i - 1, j, k)] + eb[fe.at(4, i, j, k - 1)] +
                       eb[fe.at(4, i - 1, j, k - 1)]) + b0y;
  double wbz = 0.25 * (eb[fe.at(5, i, j, k)] + eb[fe.at(5, i - 1, j, k)] + eb[fe.at(5, i, j - 1, k)] +
                       eb[fe.at(5, i - 1, j - 1, k)]) + b0z;
  f0[t] = make_float4((float)wex, (float)wey, (float)wez, (float)wbx);
  f1[t] = make_float4((float)wby, (float)wbz, 0.f, 0.f);
}

// ---------------------------------------------------------------- push
#include "fx_push.cuh"

// int64 fixed point -> FP64 field (scale 2^-40).
__global__ void k_fix_to_double(const long long* __restrict__ src, double* __restrict__ dst, int64_t n) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  dst[i] = (double)src[i] * FIX_INV;
}

// ---------------------------------------------------------------- load / store / sort
// (cell, offset) of one FP64 coordinate.  An offset that rounds up to 1.0f,
// or a coordinate exactly on the upper face x = n (left there by the
// rounding of a periodic wrap), is kept in the last cell with the largest
// FP32 offset below 1 (an error of at most 6e-8 cell).
__device__ __forceinline__ bool split_coord(double x, int n, int& c, float& o) {
  double f = floor(x);
  c = (int)f;
  o = (float)(x - f);
  const float below_one = 0.99999994f;
  if (o >= 1.0f) o = below_one;
  if (c == n && x == (double)n) { c = n - 1; o = below_one; }
  return c >= 0 && c < n;
}

__global__ void k_fx_from_aos(const emsesg_particle* __restrict__ p, int64_t n, Geo g, float4* pos, float* vx,
                              float* vy, float* vz, int* status, long long* diag) {
  int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  emsesg_particle q = p[m];
  uint32_t cell = DEAD;
  float ox = 0.f, oy = 0.f, oz = 0.f;
  if (q.nid != -1) {
    int i, j, k;
    bool ok = split_coord(q.x, g.nx, i, ox) & split_coord(q.y, g.ny, j, oy) & split_coord(q.z, g.nz, k, oz);
    if (!ok || q.preside != 0) report_bad(status, diag, SITE_FX_LOAD, m, i + 100000LL * j + 10000000000LL * k);
    else cell = pack(g, i, j, k);
  }
  pos[m] = make_float4(ox, oy, oz, __int_as_float((int)cell));
  vx[m] = (float)q.vx; vy[m] = (float)q.vy; vz[m] = (float)q.vz;
}

__global__ void k_fx_to_aos(const float4* __restrict__ pos, const float* __restrict__ vx, const float* __restrict__ vy,
                            const float* __restrict__ vz, int64_t n, Geo g, int is, emsesg_particle* p) {
  int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  float4 ps = pos[m];
  uint32_t cell = (uint32_t)__float_as_int(ps.w);
  emsesg_particle q;
  if (cell == DEAD) {
    q.x = q.y = q.z = 0.0;
    q.nid = -1;
  } else {
    int i, j, k;
    unpack(g, cell, i, j, k);
    q.x = (double)i + (double)ps.x;
    q.y = (double)j + (double)ps.y;
    q.z = (double)k + (double)ps.z;
    q.nid = 0;
  }
  q.vx = vx[m]; q.vy = vy[m]; q.vz = vz[m];
  q.pid = 0;
  q.preside = 0;
  q.spec = is + 1;
  p[m] = q;
}

// Sort key of the FP32 form: the tile-major cell key (as the FP64 spsort);
// dead particles and slots past the live count get the largest key.
__global__ void k_fx_keys(const float4* __restrict__ pos, int64_t n, const int64_t* count, Geo g, uint32_t deadkey,
                          uint32_t* keys, uint32_t* vals) {
  int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  uint32_t cell = (uint32_t)__float_as_int(pos[m].w);
  uint32_t key = deadkey;
  if (m < *count && cell != DEAD) {
    int i, j, k;
    unpack(g, cell, i, j, k);
    uint32_t tile = (uint32_t)(i / g.t[0]) + (uint32_t)g.nt[0] * ((uint32_t)(j / g.t[1]) + (uint32_t)g.nt[1] * (uint32_t)(k / g.t[2]));
    uint32_t in = (uint32_t)(i % g.t[0]) + (uint32_t)g.t[0] * ((uint32_t)(j % g.t[1]) + (uint32_t)g.t[1] * (uint32_t)(k % g.t[2]));
    key = tile * (uint32_t)(g.t[0] * g.t[1] * g.t[2]) + in;
  }
  keys[m] = key;
  vals[m] = (uint32_t)m;
}

__global__ void k_fx_gather(const float4* __restrict__ pos, const float* __restrict__ vx, const float* __restrict__ vy,
                            const float* __restrict__ vz, const uint32_t* __restrict__ idx, int64_t n, float4* pos2,
                            float* vx2, float* vy2, float* vz2) {
  int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  uint32_t s = idx[m];
  pos2[m] = pos[s];
  vx2[m] = vx[s];
  vy2[m] = vy[s];
  vz2[m] = vz[s];
}

// tile_start[t] = first sorted slot with tile >= t; tile_start[ntiles] and
// the live count = first dead slot.
__global__ void k_tile_starts(const uint32_t* __restrict__ keys, int64_t n, uint32_t tilecells, int64_t ntiles,
                              int64_t* tile_start, int64_t* count) {
  int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m > n) return;
  int64_t prev = m == 0 ? -1 : (int64_t)(keys[m - 1] / tilecells);
  int64_t cur = m == n ? ntiles : (int64_t)(keys[m] / tilecells);
  if (prev > ntiles) prev = ntiles;
  if (cur > ntiles) cur = ntiles;
  for (int64_t t = prev + 1; t <= cur; t++) tile_start[t] = m;
  if (cur == ntiles && prev < ntiles) *count = m;
}

inline unsigned nblk(int64_t n, int t = 256) { return (unsigned)std::max<int64_t>(1, (n + t - 1) / t); }

int ceil_log2(int n) {
  int b = 0;
  while ((1 << b) < n) b++;
  return std::max(b, 1);
}

Geo make_geo(emsesg_ctx* ctx) {
  const emsesg_config& c = ctx->cfg;
  Geo g;
  g.nx = c.nx; g.ny = c.ny; g.nz = c.nz;
  g.bx = ctx->fx.bits[0];
  g.by = ctx->fx.bits[1];
  g.mx = (1u << g.bx) - 1u;
  g.my = (1u << g.by) - 1u;
  for (int d = 0; d < 3; d++) { g.t[d] = ctx->fx.tile[d]; g.nt[d] = ctx->fx.ntile[d]; }
  return g;
}

}  // namespace

int fx_alloc(emsesg_ctx* ctx) {
  FxState& f = ctx->fx;
  if (f.pos) return EMSESG_OK;
  const emsesg_config& c = ctx->cfg;
  int n[3] = {c.nx, c.ny, c.nz};
  // room for cells -1 .. n shifted by +1 (the push queue keys)
  for (int d = 0; d < 3; d++) f.bits[d] = ceil_log2(n[d] + 2);
  if (f.bits[0] + f.bits[1] + f.bits[2] > 31)
    return set_error(ctx, EMSESG_ERR_ARG, "grid needs more than 31 bits of packed cell index");
  for (int d = 0; d < 3; d++) {
    int t = c.sort_tile[d] > 0 ? c.sort_tile[d] : 8;
    f.tile[d] = std::min(t, n[d]);
    f.ntile[d] = (n[d] + f.tile[d] - 1) / f.tile[d];
  }
  int tmax = std::max(f.tile[0], std::max(f.tile[1], f.tile[2]));
  if (tmax > 8) return set_error(ctx, EMSESG_ERR_ARG, "FP32 form tiles are at most 8 cells per axis");
  f.ntiles = (int64_t)f.ntile[0] * f.ntile[1] * f.ntile[2];
  int64_t cap = 0;
  for (int is = 0; is < c.nspec; is++) cap += ctx->seg.capacity[is];
  cap = std::max<int64_t>(cap, 1);
  EMSESG_CUDA(ctx, cudaMalloc(&f.pos, cap * sizeof(float4)));
  EMSESG_CUDA(ctx, cudaMalloc(&f.vx, cap * sizeof(float)));
  EMSESG_CUDA(ctx, cudaMalloc(&f.vy, cap * sizeof(float)));
  EMSESG_CUDA(ctx, cudaMalloc(&f.vz, cap * sizeof(float)));
  EMSESG_CUDA(ctx, cudaMalloc(&f.pos2, cap * sizeof(float4)));
  EMSESG_CUDA(ctx, cudaMalloc(&f.vx2, cap * sizeof(float)));
  EMSESG_CUDA(ctx, cudaMalloc(&f.vy2, cap * sizeof(float)));
  EMSESG_CUDA(ctx, cudaMalloc(&f.vz2, cap * sizeof(float)));
  EMSESG_CUDA(ctx, cudaMalloc(&f.count_d, EMSESG_ISPEC * sizeof(int64_t)));
  EMSESG_CUDA(ctx, cudaMalloc(&f.tile_start, (int64_t)c.nspec * (f.ntiles + 1) * sizeof(int64_t)));
  FieldDesc fr = field_desc(c, EMSESG_FIELD_RHO), fj = field_desc(c, EMSESG_FIELD_AJ);
  EMSESG_CUDA(ctx, cudaMalloc(&f.accum, (fr.size() + fj.size()) * sizeof(int64_t)));
  int64_t nn = (int64_t)(c.nx + 1) * (c.ny + 1) * (c.nz + 1);
  EMSESG_CUDA(ctx, cudaMalloc(&f.fnode, nn * sizeof(float4)));
  EMSESG_CUDA(ctx, cudaMalloc(&f.fnode2, nn * sizeof(float4)));
  EMSESG_CUDA(ctx, cudaFuncSetAttribute(k_fx_push<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, fx_push_smem(4)));
  EMSESG_CUDA(ctx, cudaFuncSetAttribute(k_fx_push<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, fx_push_smem(8)));
  return EMSESG_OK;
}

void fx_free(emsesg_ctx* ctx) {
  FxState& f = ctx->fx;
  cudaFree(f.pos); cudaFree(f.vx); cudaFree(f.vy); cudaFree(f.vz);
  cudaFree(f.pos2); cudaFree(f.vx2); cudaFree(f.vy2); cudaFree(f.vz2);
  cudaFree(f.count_d); cudaFree(f.tile_start); cudaFree(f.accum);
  cudaFree(f.fnode); cudaFree(f.fnode2);
  f = FxState();
}

}  // namespace emsesg

using namespace emsesg;

namespace {
int64_t max_cap(emsesg_ctx* ctx) {
  int64_t m = 0;
  for (int is = 0; is < ctx->cfg.nspec; is++) m = std::max(m, ctx->seg.capacity[is]);
  return m;
}
}  // namespace

extern "C" int emsesg_fx_sort(emsesg_ctx* ctx) {
  if (!ctx) return EMSESG_ERR_ARG;
  if (!ctx->fx.loaded) return set_error(ctx, EMSESG_ERR_STATE, "FP32 form not loaded (emsesg_fx_load)");
  int rc = ensure_sort_scratch(ctx, max_cap(ctx));
  if (rc) return rc;
  FxState& f = ctx->fx;
  Geo g = make_geo(ctx);
  uint32_t tilecells = (uint32_t)(f.tile[0] * f.tile[1] * f.tile[2]);
  uint32_t deadkey = (uint32_t)(f.ntiles * tilecells);
  int bits = 1;
  while (bits < 32 && (1ULL << bits) <= deadkey) bits++;
  for (int is = 0; is < ctx->cfg.nspec; is++) {
    int64_t n = ctx->totalp[is];  // upper bound of the live count
    int64_t off = ctx->seg.base[is];
    int64_t* ts = f.tile_start + (int64_t)is * (f.ntiles + 1);
    if (n == 0) {
      EMSESG_CUDA(ctx, cudaMemsetAsync(ts, 0, (f.ntiles + 1) * sizeof(int64_t), ctx->stream));
      EMSESG_CUDA(ctx, cudaMemsetAsync(f.count_d + is, 0, sizeof(int64_t), ctx->stream));
      continue;
    }
    EMSESG_LAUNCH(ctx, "fx_keys", k_fx_keys, nblk(n), 256, 0, f.pos + off, n, f.count_d + is, g, deadkey,
                  ctx->sort.keys[0], ctx->sort.vals[0]);
    uint32_t *ko, *vo;
    if ((rc = sort_pairs(ctx, ctx->sort.keys[0], ctx->sort.vals[0], n, bits, &ko, &vo))) return rc;
    EMSESG_LAUNCH(ctx, "fx_gather", k_fx_gather, nblk(n), 256, 0, f.pos + off, f.vx + off, f.vy + off, f.vz + off, vo,
                  n, f.pos2 + off, f.vx2 + off, f.vy2 + off, f.vz2 + off);
    EMSESG_LAUNCH(ctx, "fx_tile_starts", k_tile_starts, nblk(n + 1), 256, 0, ko, n, tilecells, f.ntiles, ts,
                  f.count_d + is);
  }
  std::swap(f.pos, f.pos2);
  std::swap(f.vx, f.vx2);
  std::swap(f.vy, f.vy2);
  std::swap(f.vz, f.vz2);
  return EMSESG_OK;
}

extern "C" int emsesg_fx_load(emsesg_ctx* ctx) {
  if (!ctx) return EMSESG_ERR_ARG;
  int rc = fx_alloc(ctx);
  if (rc) return rc;
  FxState& f = ctx->fx;
  Geo g = make_geo(ctx);
  for (int is = 0; is < ctx->cfg.nspec; is++) {
    int64_t n = ctx->totalp[is];
    int64_t off = ctx->seg.base[is];
    if (n == 0) continue;
    EMSESG_LAUNCH(ctx, "fx_from_aos", k_fx_from_aos, nblk(n), 256, 0, ctx->pbuf + off, n, g, f.pos + off, f.vx + off,
                  f.vy + off, f.vz + off, ctx->d_status, ctx->d_diag);
  }
  EMSESG_CUDA(ctx, cudaMemcpyAsync(f.count_d, ctx->totalp, EMSESG_ISPEC * sizeof(int64_t), cudaMemcpyHostToDevice,
                                   ctx->stream));
  f.loaded = true;
  rc = emsesg_fx_sort(ctx);
  if (rc) return rc;
  return emsesg_synchronize(ctx);
}

extern "C" int emsesg_fx_counts(emsesg_ctx* ctx, int64_t* totalp) {
  if (!ctx || !totalp) return EMSESG_ERR_ARG;
  if (!ctx->fx.loaded) return set_error(ctx, EMSESG_ERR_STATE, "FP32 form not loaded");
  EMSESG_CUDA(ctx, cudaMemcpyAsync(totalp, ctx->fx.count_d, ctx->cfg.nspec * sizeof(int64_t), cudaMemcpyDeviceToHost,
                                   ctx->stream));
  EMSESG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return EMSESG_OK;
}

extern "C" int emsesg_fx_store(emsesg_ctx* ctx) {
  if (!ctx) return EMSESG_ERR_ARG;
  if (!ctx->fx.loaded) return set_error(ctx, EMSESG_ERR_STATE, "FP32 form not loaded");
  // Current buffer order; particles that died since the last sort come out
  // with nid = -1 in place, as the reference leaves them before transbound.
  int64_t cnt[EMSESG_ISPEC] = {0};
  int rc = emsesg_fx_counts(ctx, cnt);
  if (rc) return rc;
  FxState& f = ctx->fx;
  Geo g = make_geo(ctx);
  for (int is = 0; is < ctx->cfg.nspec; is++) {
    int64_t off = ctx->seg.base[is];
    ctx->totalp[is] = cnt[is];
    if (cnt[is] == 0) continue;
    EMSESG_LAUNCH(ctx, "fx_to_aos", k_fx_to_aos, nblk(cnt[is]), 256, 0, f.pos + off, f.vx + off, f.vy + off,
                  f.vz + off, cnt[is], g, is, ctx->pbuf + off);
  }
  EMSESG_CUDA(ctx, cudaMemcpyAsync(ctx->d_count, ctx->totalp, EMSESG_ISPEC * sizeof(int64_t), cudaMemcpyHostToDevice,
                                   ctx->stream));
  return emsesg_synchronize(ctx);
}

extern "C" int emsesg_fx_step(emsesg_ctx* ctx, int ustep, int do_sort) {
  if (!ctx) return EMSESG_ERR_ARG;
  if (!ctx->fx.loaded) return set_error(ctx, EMSESG_ERR_STATE, "FP32 form not loaded (emsesg_fx_load)");
  if (ustep < 1) return set_error(ctx, EMSESG_ERR_ARG, "ustep must be >= 1");
  const emsesg_config& c = ctx->cfg;
  if (c.npc > 0 && c.line_mode != 1)
    return set_error(ctx, EMSESG_ERR_UNSUPPORTED, "the FP32 form has no body absorption yet");
  int rc;
  if (do_sort && (rc = emsesg_fx_sort(ctx))) return rc;
  FxState& f = ctx->fx;
  Geo g = make_geo(ctx);
  int64_t nn = (int64_t)(c.nx + 1) * (c.ny + 1) * (c.nz + 1);
  EMSESG_LAUNCH(ctx, "fx_grdcrt", k_grdcrt32, nblk(nn), 256, 0, ctx->field[EMSESG_FIELD_EB], f.fnode, f.fnode2,
                field_desc(c, EMSESG_FIELD_EB), c.nx, c.ny, c.nz, c.e0[0], c.e0[1], c.e0[2], c.b0[0], c.b0[1],
                c.b0[2]);
  FieldDesc fr = field_desc(c, EMSESG_FIELD_RHO), fj = field_desc(c, EMSESG_FIELD_AJ);
  unsigned long long* acc_rho = (unsigned long long*)f.accum;
  unsigned long long* acc_j = acc_rho + fr.size();
  EMSESG_CUDA(ctx, cudaMemsetAsync(f.accum, 0, (fr.size() + fj.size()) * sizeof(int64_t), ctx->stream));
  int tmax = std::max(f.tile[0], std::max(f.tile[1], f.tile[2]));
  int smem = fx_push_smem(tmax);
  FxPushArgs a{};
  a.pos = f.pos; a.vx = f.vx; a.vy = f.vy; a.vz = f.vz;
  a.tile_start = f.tile_start;
  a.ntiles = f.ntiles;
  double gustep = ustep;
  a.gustep = (float)gustep;
  a.rustep = (float)(1.0 / ustep);
  for (int is = 0; is < c.nspec; is++) {
    a.off[is] = ctx->seg.base[is];
    for (int d = 0; d < 3; d++) a.npbnd[is][d] = c.npbnd[is][d];
    a.qmp[is] = (float)(c.qm[is] * gustep * 0.5);
    a.qfix[is] = (float)(c.q[is] * 1099511627776.0);
  }
  a.f0 = f.fnode; a.f1 = f.fnode2;
  a.acc_rho = acc_rho; a.acc_j = acc_j;
  a.fr = fr; a.fj = fj;
  a.g = g;
  a.nesc = ctx->d_counter->nesc;
  a.status = ctx->d_status;
  a.diag = ctx->d_diag;
  dim3 grid((unsigned)f.ntiles, (unsigned)c.nspec);
  if (fx_box_tile(tmax) == 4)
    EMSESG_LAUNCH(ctx, "fx_push", k_fx_push<4>, grid, PUSH_THREADS, smem, a);
  else
    EMSESG_LAUNCH(ctx, "fx_push", k_fx_push<8>, grid, PUSH_THREADS, smem, a);
  // guard folding on the exact integers, then FP64 outputs
  if ((rc = run_slab_ops(ctx, (long long*)acc_rho, fr, fold_ops(c, 0, 1), "fx_fold_rho"))) return rc;
  if ((rc = run_slab_ops(ctx, (long long*)acc_j, fj, fold_ops(c, 1, 3), "fx_fold_j"))) return rc;
  EMSESG_LAUNCH(ctx, "fx_to_double", k_fix_to_double, nblk(fr.size()), 256, 0, (const long long*)acc_rho,
                ctx->field[EMSESG_FIELD_RHO], fr.size());
  EMSESG_LAUNCH(ctx, "fx_to_double", k_fix_to_double, nblk(fj.size()), 256, 0, (const long long*)acc_j,
                ctx->field[EMSESG_FIELD_AJ], fj.size());
  ctx->rng_stream++;
  return EMSESG_OK;
}

extern "C" int emsesg_fx_download_accum(emsesg_ctx* ctx, int64_t* host) {
  if (!ctx || !host) return EMSESG_ERR_ARG;
  if (!ctx->fx.accum) return set_error(ctx, EMSESG_ERR_STATE, "FP32 form not loaded");
  FieldDesc fr = field_desc(ctx->cfg, EMSESG_FIELD_RHO), fj = field_desc(ctx->cfg, EMSESG_FIELD_AJ);
  EMSESG_CUDA(ctx, cudaMemcpyAsync(host, ctx->fx.accum, (fr.size() + fj.size()) * sizeof(int64_t),
                                   cudaMemcpyDeviceToHost, ctx->stream));
  EMSESG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return EMSESG_OK;
}
