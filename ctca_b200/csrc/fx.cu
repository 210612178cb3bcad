// fx.cu -- the FP32 / fixed-point form of the EMSES particle step.
//
// Particle state (per species region, 28 bytes a particle):
//   pos[m] = {ox, oy, oz, cell}: in-cell offsets in [0,1) (FP32) and the
//            packed cell index i | j<<bx | k<<(bx+by) (int32 bits; all ones
//            marks a dead particle),
//   vx[m], vy[m], vz[m]: FP32 velocities in internal units.
// Particles stay sorted by the tile-major cell key (8x8x8 cell tiles by
// default): tile_start[t] .. tile_start[t+1] are the sorted ranks of tile t
// at the last sort, stored thread-major in the padded slot region that starts
// at tile_pad[t] (fx_push.cuh), and one CTA pushes one tile of one species.
//
// The step kernel fuses, per particle: the trilinear E/B gather from the
// FP32 node field (grdcrt output), the Buneman-Boris push, the move and the
// outer boundary rules of psolve1.F90:366-606 evaluated on (integer cell,
// FP32 offset) pairs, the zigzag current of psolve1.F90:717-789 and the CIC
// charge of charge.F90:59-80 at the new position (fx_push.cuh).  Deposits
// are summed per cell in registers along each thread's sorted slice,
// converted to int64 fixed point at 2^40 and added into a shared-memory
// accumulator covering the tile plus a 1-cell guard; the CTA then adds its
// accumulator into the global int64 arrays.  Integer adds commute, so the
// global sums do not depend on the order in which CTAs and atomics run, and
// the FP32 partial sums depend only on the sorted order and the fixed thread
// slicing, so every run gives the same bits.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>
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
// nodes 0..n on the x and y axes, node planes k0 .. k0 + nk - 1 on z (node
// plane k reads the eb planes k - 1 and k).
__global__ void k_grdcrt32(const double* __restrict__ eb, float4* __restrict__ f0, float4* __restrict__ f1,
                           FieldDesc fe, int nx, int ny, int k0, int nk, double e0x, double e0y, double e0z,
                           double b0x, double b0y, double b0z) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t ex = nx + 1, ey = ny + 1;
  if (t >= ex * ey * nk) return;
  int i = (int)(t % ex), j = (int)((t / ex) % ey), k = k0 + (int)(t / (ex * ey));
  t += (int64_t)k0 * ex * ey;
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

// One tile region (thread-major, see fx_push.cuh) back to the FP64 records
// of the tile's sorted ranks ts[t] .. ts[t+1]-1.
// Injected records into the tail zone (oh2_inject_particle, ohhelp2.c:549):
// preside +1 takes a random fraction of its first step (ord > 0), an
// anti-particle (preside -2, an emitted particle's image on the body face,
// psuper3.F90:203-206) removes one count from the surface cell it lies on
// and takes no slot's place in the push (DEAD).
__global__ void k_fx_inject(const emsesg_particle* __restrict__ q, const int32_t* __restrict__ qord, int64_t n,
                            Geo g, Bodies bd, int64_t slot0, float4* pos, float* vx, float* vy, float* vz,
                            int32_t* ord, unsigned long long* surf, int* status, long long* diag) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const emsesg_particle r = q[k];
  const int64_t m = slot0 + k;
  uint32_t cell = DEAD;
  float ox = 0.f, oy = 0.f, oz = 0.f;
  if (r.preside == EMSESG_PCL_TO_BE_ACCUMULATED_AS_ANTIPCL) {
    const double p3[3] = {r.x, r.y, r.z};
    for (int b = 0; b < bd.n; b++) {
      if (bd.kind[b] != 0) continue;  // surface cells of box bodies only
      int64_t hit = -1;
      for (int d = 0; d < 3 && hit < 0; d++) {
        const int e1 = d == 0 ? 1 : 0, e2 = d == 2 ? 1 : 2;
        if (p3[e1] < bd.lo[b][e1] || p3[e1] > bd.hi[b][e1] || p3[e2] < bd.lo[b][e2] || p3[e2] > bd.hi[b][e2]) continue;
        int side = -1;
        if (p3[d] == (double)bd.lo[b][d]) side = 0;
        else if (p3[d] == (double)bd.hi[b][d]) side = 1;
        if (side < 0) continue;
        int u = (int)floor(p3[e1]), v = (int)floor(p3[e2]);
        u = min(max(u, bd.lo[b][e1]), bd.hi[b][e1] - 1) - bd.lo[b][e1];
        v = min(max(v, bd.lo[b][e2]), bd.hi[b][e2] - 1) - bd.lo[b][e2];
        hit = bd.off[b][2 * d + side] + u + (int64_t)(bd.hi[b][e1] - bd.lo[b][e1]) * v;
      }
      if (hit >= 0) {
        atomicAdd(&surf[hit], (unsigned long long)(-1LL));
        break;
      }
    }
  } else if (r.nid != -1) {
    int i, j, kk;
    bool ok = split_coord(r.x, g.nx, i, ox) & split_coord(r.y, g.ny, j, oy) & split_coord(r.z, g.nz, kk, oz);
    if (!ok) report_bad(status, diag, SITE_FX_LOAD, m, i + 100000LL * j + 10000000000LL * kk);
    else cell = pack(g, i, j, kk);
  }
  pos[m] = make_float4(ox, oy, oz, __int_as_float((int)cell));
  vx[m] = (float)r.vx;
  vy[m] = (float)r.vy;
  vz[m] = (float)r.vz;
  ord[k] = cell == DEAD ? 0 : qord[k];
}

// chgacm += influx * q * sqdscaled for conductors (psolve1.F90:821-828).
__global__ void k_fx_chgacm(const emsesg_config* c, emsesg_counter* gc) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int is = 0; is < c->nspec; is++)
    for (int ipc = 0; ipc < c->npc; ipc++)
      if (c->body[ipc].ncond > 0) {
        double add = (double)gc->influx[is][ipc] * c->q[is] * c->body[ipc].sqdscaled;
        gc->chgacm[ipc][0] = gc->chgacm[ipc][0] + add;
        gc->chgacm[ipc][1] = gc->chgacm[ipc][1] + add;
      }
}

__global__ void k_add_i64(int64_t* p, int64_t v) { *p += v; }

__global__ void k_fx_to_aos_tm(const float4* __restrict__ pos, const float* __restrict__ vx,
                               const float* __restrict__ vy, const float* __restrict__ vz,
                               const int64_t* __restrict__ ts, const int64_t* __restrict__ tp, Geo g, int is,
                               emsesg_particle* p) {
  const int t = blockIdx.x, tid = threadIdx.x;
  const int64_t n = ts[t + 1] - ts[t];
  if (n <= 0) return;
  const int L = (int)((n + PUSH_THREADS - 1) / PUSH_THREADS);
  for (int r = 0; r < L; r++) {
    const int64_t q = (int64_t)tid * L + r;
    if (q >= n) continue;
    const int64_t m = tp[t] + (int64_t)r * PUSH_THREADS + tid;
    float4 ps = pos[m];
    uint32_t cell = (uint32_t)__float_as_int(ps.w);
    emsesg_particle o;
    if (cell == DEAD) {
      o.x = o.y = o.z = 0.0;
      o.nid = -1;
    } else {
      int i, j, k;
      unpack(g, cell, i, j, k);
      o.x = (double)i + (double)ps.x;
      o.y = (double)j + (double)ps.y;
      o.z = (double)k + (double)ps.z;
      o.nid = 0;
    }
    o.vx = vx[m]; o.vy = vy[m]; o.vz = vz[m];
    o.pid = 0;
    o.preside = 0;
    o.spec = is + 1;
    p[ts[t] + q] = o;
  }
}

// Sort key of the FP32 form: the tile-major cell key (as the FP64 spsort);
// dead particles, empty slots and slots past the region's slot count get the
// largest key.
__global__ void k_fx_keys(const float4* __restrict__ pos, int64_t n, const int64_t* slots, int64_t tail0,
                          int64_t ntail, Geo g, uint32_t deadkey, uint32_t* keys, uint32_t* vals) {
  int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n + ntail) return;
  uint32_t key = deadkey;
  // indices past n are the tail zone's slots
  const int64_t slot = m < n ? m : tail0 + (m - n);
  if (m >= n || m < *slots) {
    uint32_t cell = (uint32_t)__float_as_int(pos[slot].w);
    if (cell != DEAD) {
      int i, j, k;
      unpack(g, cell, i, j, k);
      uint32_t tile = (uint32_t)(i / g.t[0]) +
                      (uint32_t)g.nt[0] * ((uint32_t)(j / g.t[1]) + (uint32_t)g.nt[1] * (uint32_t)(k / g.t[2]));
      uint32_t in = (uint32_t)(i % g.t[0]) + (uint32_t)g.t[0] * ((uint32_t)(j % g.t[1]) + (uint32_t)g.t[1] * (uint32_t)(k % g.t[2]));
      key = tile * (uint32_t)(g.t[0] * g.t[1] * g.t[2]) + in;
    }
  }
  keys[m] = key;
  vals[m] = (uint32_t)slot;
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

// Padded region starts: tile t gets ceil(n_t / PUSH_THREADS) full rows.  One
// block of 1024 threads scans the ntiles counts; slots = total.
__global__ void __launch_bounds__(1024) k_tile_pad(const int64_t* __restrict__ ts, int64_t ntiles, int64_t* tp,
                                                   int64_t* slots) {
  __shared__ int64_t part[1024];
  const int tid = threadIdx.x;
  const int64_t per = (ntiles + 1023) / 1024;
  const int64_t t0 = tid * per, t1 = min(ntiles, t0 + per);
  int64_t sum = 0;
  for (int64_t t = t0; t < t1; t++) {
    int64_t n = ts[t + 1] - ts[t];
    sum += (n + PUSH_THREADS - 1) / PUSH_THREADS * PUSH_THREADS;
  }
  part[tid] = sum;
  __syncthreads();
  for (int d = 1; d < 1024; d <<= 1) {
    int64_t v = tid >= d ? part[tid - d] : 0;
    __syncthreads();
    part[tid] += v;
    __syncthreads();
  }
  int64_t run = part[tid] - sum;  // exclusive prefix of this thread's chunk
  for (int64_t t = t0; t < t1; t++) {
    tp[t] = run;
    int64_t n = ts[t + 1] - ts[t];
    run += (n + PUSH_THREADS - 1) / PUSH_THREADS * PUSH_THREADS;
  }
  if (tid == 1023) {
    tp[ntiles] = part[1023];
    *slots = part[1023];
  }
}

// Sorted ranks -> thread-major tile regions (fx_push.cuh): slot
// tp[t] + r*PUSH_THREADS + c holds rank ts[t] + c*L + r; empty slots get a
// DEAD cell.  One block per tile, coalesced writes.
__global__ void k_fx_gather_tm(const float4* __restrict__ pos, const float* __restrict__ vx,
                               const float* __restrict__ vy, const float* __restrict__ vz,
                               const uint32_t* __restrict__ idx, const int64_t* __restrict__ ts,
                               const int64_t* __restrict__ tp, float4* pos2, float* vx2, float* vy2, float* vz2,
                               uint32_t* inv) {
  const int t = blockIdx.x, tid = threadIdx.x;
  const int64_t n = ts[t + 1] - ts[t];
  if (n <= 0) return;
  const int L = (int)((n + PUSH_THREADS - 1) / PUSH_THREADS);
  for (int r = 0; r < L; r++) {
    const int64_t q = (int64_t)tid * L + r;
    const int64_t m = tp[t] + (int64_t)r * PUSH_THREADS + tid;
    if (q < n) {
      const uint32_t src = idx[ts[t] + q];
      pos2[m] = pos[src];
      vx2[m] = vx[src];
      vy2[m] = vy[src];
      vz2[m] = vz[src];
      inv[m] = src;
    } else {
      pos2[m] = make_float4(0.f, 0.f, 0.f, __int_as_float((int)DEAD));
      vx2[m] = 0.f;
      vy2[m] = 0.f;
      vz2[m] = 0.f;
      inv[m] = DEAD;
    }
  }
}

#include "fx_sort.cuh"
#include "fx_adjoint.cuh"
#include "fx_diag.cuh"

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

// Bodies usable by the FP32 form: boxes (geotype 0/1) with integer bounds,
// cylinders (geotype 2, axis 1..3) and spheres (geotype 3) of positive
// radius.  Returns false (with the reason) when a body cannot be handled.
bool bodies_supported(const emsesg_config& c, std::string* why) {
  if (c.npc <= 0 || c.line_mode == 1) return true;
  for (int ipc = 0; ipc < c.npc; ipc++) {
    const emsesg_body& b = c.body[ipc];
    if (b.geotype == 2 || b.geotype == 3) {
      if (!(b.radius > 0.0) || (b.geotype == 2 && (b.cyl_align < 1 || b.cyl_align > 3))) {
        if (why) *why = "cylinder or sphere body without a positive radius or a valid axis";
        return false;
      }
      continue;
    }
    if (!(b.geotype == 0 || b.geotype == 1)) {
      if (why) *why = "the FP32 form handles box, cylinder and sphere bodies (geotype 0..3) only";
      return false;
    }
    const double v[6] = {b.xlpc, b.xupc, b.ylpc, b.yupc, b.zlpc, b.zupc};
    for (int q = 0; q < 6; q++)
      if (v[q] != std::floor(v[q])) {
        if (why) *why = "the FP32 form needs integer box bounds";
        return false;
      }
    if (!(b.xupc > b.xlpc && b.yupc > b.ylpc && b.zupc > b.zlpc)) {
      if (why) *why = "empty box body";
      return false;
    }
  }
  return true;
}

Bodies make_bodies(const emsesg_config& c) {
  Bodies bd{};
  bd.n = 0;
  bd.nsurf = 0;
  if (c.line_mode == 1 || !bodies_supported(c, nullptr)) return bd;
  for (int ipc = 0; ipc < c.npc; ipc++) {
    const emsesg_body& b = c.body[ipc];
    const int q = bd.n++;
    bd.ipc[q] = ipc;
    if (b.geotype == 2 || b.geotype == 3) {
      // the cells a point inside may lie in, with one cell of margin
      double lo[3], hi[3];
      if (b.geotype == 3) {
        for (int d = 0; d < 3; d++) {
          bd.cen[q][d] = (float)b.sph_center[d];
          lo[d] = b.sph_center[d] - b.radius;
          hi[d] = b.sph_center[d] + b.radius;
        }
      } else {
        const int a0 = b.cyl_align - 1, a1 = (a0 + 1) % 3, a2 = (a0 + 2) % 3;
        bd.cax[q] = a0;
        bd.cen[q][a0] = 0.f;
        bd.cen[q][a1] = (float)b.cyl_axis[0];
        bd.cen[q][a2] = (float)b.cyl_axis[1];
        bd.edge[q][0] = (float)b.cyl_edge[0];
        bd.edge[q][1] = (float)b.cyl_edge[1];
        lo[a0] = b.cyl_edge[0]; hi[a0] = b.cyl_edge[1];
        lo[a1] = b.cyl_axis[0] - b.radius; hi[a1] = b.cyl_axis[0] + b.radius;
        lo[a2] = b.cyl_axis[1] - b.radius; hi[a2] = b.cyl_axis[1] + b.radius;
      }
      bd.kind[q] = b.geotype;
      bd.r2[q] = (float)(b.radius * b.radius);
      for (int d = 0; d < 3; d++) {
        bd.lo[q][d] = (int)std::max(-2.0, std::floor(lo[d]) - 1.0);
        bd.hi[q][d] = (int)std::min(1e9, std::floor(hi[d]) + 1.0);
      }
      for (int f = 0; f < 6; f++) bd.off[q][f] = -1;
      bd.ncurved++;
      continue;
    }
    bd.kind[q] = 0;
    bd.lo[q][0] = (int)b.xlpc; bd.hi[q][0] = (int)b.xupc;
    bd.lo[q][1] = (int)b.ylpc; bd.hi[q][1] = (int)b.yupc;
    bd.lo[q][2] = (int)b.zlpc; bd.hi[q][2] = (int)b.zupc;
    for (int f = 0; f < 6; f++) {
      const int d = f / 2, e1 = d == 0 ? 1 : 0, e2 = d == 2 ? 1 : 2;
      bd.off[q][f] = bd.nsurf;
      bd.nsurf += (int64_t)(bd.hi[q][e1] - bd.lo[q][e1]) * (bd.hi[q][e2] - bd.lo[q][e2]);
    }
  }
  return bd;
}

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
  // species regions: capacity plus one row of padding per tile, in whole
  // rows, then the tail zone of injected particles (an eighth of capacity)
  int64_t cap = 0, ntailall = 0;
  for (int is = 0; is < c.nspec; is++) {
    f.base[is] = cap;
    int64_t rows = (ctx->seg.capacity[is] + PUSH_THREADS - 1) / PUSH_THREADS + f.ntiles;
    f.tail0[is] = rows * PUSH_THREADS;
    f.tailcap[is] = ((ctx->seg.capacity[is] / 8 + PUSH_THREADS - 1) / PUSH_THREADS + 1) * PUSH_THREADS;
    f.tailord_base[is] = ntailall;
    ntailall += f.tailcap[is];
    f.ntail[is] = 0;
    f.pending[is] = 0;
    f.cap[is] = f.tail0[is] + f.tailcap[is];
    cap += f.cap[is];
  }
  cap = std::max<int64_t>(cap, 1);
  EMSESG_CUDA(ctx, cudaMalloc(&f.tailord, std::max<int64_t>(ntailall, 1) * sizeof(int32_t)));
  EMSESG_CUDA(ctx, cudaMemsetAsync(f.tailord, 0, std::max<int64_t>(ntailall, 1) * sizeof(int32_t), ctx->stream));
  {
    Bodies bd = make_bodies(c);
    f.nsurf = bd.nsurf;
    const int64_t ns = std::max<int64_t>((int64_t)c.nspec * f.nsurf, 1);
    EMSESG_CUDA(ctx, cudaMalloc(&f.surf, ns * sizeof(unsigned long long)));
    EMSESG_CUDA(ctx, cudaMemsetAsync(f.surf, 0, ns * sizeof(unsigned long long), ctx->stream));
  }
  EMSESG_CUDA(ctx, cudaMalloc(&f.pos, cap * sizeof(float4)));
  EMSESG_CUDA(ctx, cudaMalloc(&f.vx, cap * sizeof(float)));
  EMSESG_CUDA(ctx, cudaMalloc(&f.vy, cap * sizeof(float)));
  EMSESG_CUDA(ctx, cudaMalloc(&f.vz, cap * sizeof(float)));
  EMSESG_CUDA(ctx, cudaMalloc(&f.pos2, cap * sizeof(float4)));
  EMSESG_CUDA(ctx, cudaMalloc(&f.vx2, cap * sizeof(float)));
  EMSESG_CUDA(ctx, cudaMalloc(&f.vy2, cap * sizeof(float)));
  EMSESG_CUDA(ctx, cudaMalloc(&f.vz2, cap * sizeof(float)));
  EMSESG_CUDA(ctx, cudaMalloc(&f.count_d, EMSESG_ISPEC * sizeof(int64_t)));
  EMSESG_CUDA(ctx, cudaMalloc(&f.slots_d, EMSESG_ISPEC * sizeof(int64_t)));
  EMSESG_CUDA(ctx, cudaMalloc(&f.tile_start, (int64_t)c.nspec * (f.ntiles + 1) * sizeof(int64_t)));
  EMSESG_CUDA(ctx, cudaMalloc(&f.tile_pad, (int64_t)c.nspec * (f.ntiles + 1) * sizeof(int64_t)));
  EMSESG_CUDA(ctx, cudaMalloc(&f.chunk_start, (int64_t)c.nspec * (f.ntiles + 1) * sizeof(int64_t)));
  FieldDesc fr = field_desc(c, EMSESG_FIELD_RHO), fj = field_desc(c, EMSESG_FIELD_AJ);
  EMSESG_CUDA(ctx, cudaMalloc(&f.accum, (fr.size() + fj.size()) * sizeof(int64_t)));
  // one bit per slot: the particles the parts of a step leave for k_fx_deferred
  f.defer_words = (cap + 31) / 32;
  EMSESG_CUDA(ctx, cudaMalloc(&f.defer, f.defer_words * sizeof(uint32_t)));
  EMSESG_CUDA(ctx, cudaMemsetAsync(f.defer, 0, f.defer_words * sizeof(uint32_t), ctx->stream));
  // FP64 checks: energy partials and sums, the continuity maxima
  EMSESG_CUDA(ctx, cudaMalloc(&f.diag, (3 * DIAG_GRID + 3 + 2) * sizeof(double)));
  EMSESG_CUDA(ctx, cudaMemsetAsync(f.diag, 0, (3 * DIAG_GRID + 3 + 2) * sizeof(double), ctx->stream));
  int64_t nn = (int64_t)(c.nx + 1) * (c.ny + 1) * (c.nz + 1);
  EMSESG_CUDA(ctx, cudaMalloc(&f.fnode, nn * sizeof(float4)));
  EMSESG_CUDA(ctx, cudaMalloc(&f.fnode2, nn * sizeof(float4)));
  // tile-local sort scratch (tiles of at most 8 cells a side)
  {
    const int64_t nbc = (int64_t)(f.tile[0] + 2) * (f.tile[1] + 2) * (f.tile[2] + 2);
    const int64_t tcells = (int64_t)f.tile[0] * f.tile[1] * f.tile[2];
    const int64_t ns = c.nspec;
    EMSESG_CUDA(ctx, cudaMalloc(&f.tile_start2, ns * (f.ntiles + 1) * sizeof(int64_t)));
    EMSESG_CUDA(ctx, cudaMalloc(&f.tile_pad2, ns * (f.ntiles + 1) * sizeof(int64_t)));
    EMSESG_CUDA(ctx, cudaMalloc(&f.lcs_cnt, ns * f.ntiles * nbc * sizeof(uint32_t)));
    EMSESG_CUDA(ctx, cudaMalloc(&f.lcs_base, ns * f.ntiles * nbc * sizeof(uint32_t)));
    EMSESG_CUDA(ctx, cudaMalloc(&f.lcs_wcnt, f.ntiles * PUSH_WARPS * nbc * sizeof(uint32_t)));  // one species
    EMSESG_CUDA(ctx, cudaMalloc(&f.lcs_celltot, f.ntiles * tcells * sizeof(uint32_t)));
    EMSESG_CUDA(ctx, cudaMalloc(&f.lcs_tiletot, f.ntiles * sizeof(int64_t)));
    EMSESG_CUDA(ctx, cudaMalloc(&f.lcs_stray, EMSESG_ISPEC * sizeof(int)));
    EMSESG_CUDA(ctx, cudaMalloc(&f.lcs_inv, cap * sizeof(uint32_t)));
    // kernel attributes hold for every context of the process: allow the
    // largest box (8-cell tiles), whatever this context's tile
    const int lsm = (int)(PUSH_WARPS * 10 * 10 * 10 * sizeof(uint32_t));
    EMSESG_CUDA(ctx, cudaFuncSetAttribute(k_lcs_count, cudaFuncAttributeMaxDynamicSharedMemorySize, lsm));
    EMSESG_CUDA(ctx, cudaFuncSetAttribute(k_lcs_rank, cudaFuncAttributeMaxDynamicSharedMemorySize, lsm));
    EMSESG_CUDA(ctx, cudaFuncSetAttribute(k_lcs_move<MoveBig>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          move_smem<MoveBig>()));
    EMSESG_CUDA(ctx, cudaFuncSetAttribute(k_lcs_move<MoveSmall>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          move_smem<MoveSmall>()));
    EMSESG_CUDA(ctx, cudaFuncSetAttribute(k_lcs_move<MoveMid>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          move_smem<MoveMid>()));
  }
  EMSESG_CUDA(ctx, cudaFuncSetAttribute(k_fx_push<4, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        fx_push_smem(4)));
  EMSESG_CUDA(ctx, cudaFuncSetAttribute(k_fx_push<8, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        fx_push_smem(8)));
  for (int box : {4, 8})
    for (int curved = 0; curved < 2; curved++)
      for (int jd = 0; jd < 2; jd++)
        for (int parts = 0; parts < 2; parts++)
          EMSESG_CUDA(ctx, cudaFuncSetAttribute(push_kernel(box, curved != 0, jd != 0, parts != 0),
                                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                fx_push_smem(box, jd != 0)));
  return EMSESG_OK;
}

void fx_free(emsesg_ctx* ctx) {
  FxState& f = ctx->fx;
  cudaFree(f.pos); cudaFree(f.vx); cudaFree(f.vy); cudaFree(f.vz);
  cudaFree(f.pos2); cudaFree(f.vx2); cudaFree(f.vy2); cudaFree(f.vz2);
  cudaFree(f.count_d); cudaFree(f.slots_d); cudaFree(f.tile_start); cudaFree(f.tile_pad); cudaFree(f.accum);
  cudaFree(f.chunk_start); cudaFree(f.defer);
  cudaFree(f.fnode); cudaFree(f.fnode2);
  cudaFree(f.diag);
  cudaFree(f.tile_start2); cudaFree(f.tile_pad2); cudaFree(f.lcs_cnt); cudaFree(f.lcs_base); cudaFree(f.lcs_wcnt);
  cudaFree(f.lcs_celltot); cudaFree(f.lcs_tiletot); cudaFree(f.lcs_stray); cudaFree(f.lcs_inv);
  cudaFree(f.surf); cudaFree(f.tailord); cudaFree(f.stage); cudaFree(f.stage_ord);
  cudaFreeHost(f.ord_host);
  if (f.ord_ev) cudaEventDestroy(f.ord_ev);
  cudaFree(f.inj_tab);
  cudaFree(f.outbox); cudaFree(f.outbox2); cudaFree(f.outbox_n);
  if (f.gexec) cudaGraphExecDestroy(f.gexec);
  adj_free(f);
  f = FxState();
}

}  // namespace emsesg

using namespace emsesg;

namespace {
// Host-side bound of the slots the sort has to look at: the particles loaded
// (no particle is added in this form) plus the padding, within the region.
int64_t sort_slots(emsesg_ctx* ctx, int is) {
  return std::min(ctx->fx.tail0[is], ctx->totalp[is] + ctx->fx.ntiles * PUSH_THREADS);
}
}  // namespace

// The tile-local counting sort (fx_sort.cuh).  Sets *done = false, having
// changed nothing, when a particle left its tile's sort box; the caller then
// sorts with the radix path.
int fx_local_sort(emsesg_ctx* ctx, bool* done) {
  *done = false;
  FxState& f = ctx->fx;
  const emsesg_config& c = ctx->cfg;
  Geo g = make_geo(ctx);
  LcsGeo G[EMSESG_ISPEC] = {};
  const int n[3] = {c.nx, c.ny, c.nz};
  for (int is = 0; is < c.nspec; is++) {
    G[is].nbc = 1;
    G[is].tcells = 1;
    for (int d = 0; d < 3; d++) {
      G[is].n[d] = n[d];
      G[is].t[d] = f.tile[d];
      G[is].nt[d] = f.ntile[d];
      G[is].bc[d] = f.tile[d] + 2;
      G[is].nbc *= G[is].bc[d];
      G[is].tcells *= f.tile[d];
      G[is].wrap[d] = c.npbnd[is][d] == 0;
    }
  }
  const int64_t nbc = G[0].nbc;
  const int lsm = (int)(PUSH_WARPS * nbc * sizeof(uint32_t));
  const int64_t T1 = f.ntiles + 1;
  // injected particles of the tail zones: sorted alone by cell key
  const uint32_t tcells = (uint32_t)(f.tile[0] * f.tile[1] * f.tile[2]);
  const uint32_t deadkey = (uint32_t)(f.ntiles * tcells);
  int kbits = 1;
  while (kbits < 32 && (1ULL << kbits) <= deadkey) kbits++;
  {
    int64_t most = 0;
    for (int is = 0; is < c.nspec; is++) most = std::max(most, f.ntail[is]);
    if (most > 0) {
      int rc = ensure_sort_scratch(ctx, most);
      if (rc) return rc;
    }
  }
  EMSESG_CUDA(ctx, cudaMemsetAsync(f.lcs_stray, 0, EMSESG_ISPEC * sizeof(int), ctx->stream));
  for (int is = 0; is < c.nspec; is++) {
    int64_t* ts2 = f.tile_start2 + is * T1;
    int64_t* tp2 = f.tile_pad2 + is * T1;
    if (ctx->totalp[is] == 0) {
      EMSESG_CUDA(ctx, cudaMemsetAsync(ts2, 0, T1 * sizeof(int64_t), ctx->stream));
      EMSESG_CUDA(ctx, cudaMemsetAsync(tp2, 0, T1 * sizeof(int64_t), ctx->stream));
      EMSESG_CUDA(ctx, cudaMemsetAsync(f.count_d + is, 0, sizeof(int64_t), ctx->stream));
      EMSESG_CUDA(ctx, cudaMemsetAsync(f.slots_d + is, 0, sizeof(int64_t), ctx->stream));
      continue;
    }
    const int64_t off = f.base[is];
    uint32_t* cnt = f.lcs_cnt + is * f.ntiles * nbc;
    uint32_t* bas = f.lcs_base + is * f.ntiles * nbc;
    const int* stray = f.lcs_stray + is;
    // per-warp counts (one species at a time)
    EMSESG_LAUNCH(ctx, "lcs_count", k_lcs_count, (unsigned)f.ntiles, PUSH_THREADS, lsm, f.pos + off,
                  f.tile_start + is * T1, f.tile_pad + is * T1, g, G[is], f.lcs_wcnt, cnt, f.lcs_stray + is);
    // Outside a stream capture the host reads the stray flag and falls back
    // to the radix sort (which redoes every species).  Inside one
    // (emsesg_fx_run's graph) it cannot: the sort kernels of a species with
    // a stray then return at once and k_lcs_keep carries its current order
    // over to the new buffers.
    if (!f.capture) {
      int st = 0;
      EMSESG_CUDA(ctx, cudaMemcpyAsync(&st, f.lcs_stray + is, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
      EMSESG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
      if (st) return EMSESG_OK;
    }
    // the species' tail zone, sorted by cell key
    const int64_t nt = f.ntail[is];
    uint32_t *tk = nullptr, *tv = nullptr;
    if (nt > 0) {
      EMSESG_LAUNCH(ctx, "lcs_tail_keys", k_fx_keys, nblk(nt), 256, 0, f.pos + off, (int64_t)0, f.slots_d + is,
                    f.tail0[is], nt, g, deadkey, ctx->sort.keys[0], ctx->sort.vals[0]);
      int rc = sort_pairs(ctx, ctx->sort.keys[0], ctx->sort.vals[0], nt, kbits, &tk, &tv);
      if (rc) return rc;
    }
    EMSESG_LAUNCH(ctx, "lcs_celltot", k_lcs_celltot, (unsigned)f.ntiles, CELL_THREADS, 0, cnt, g, G[is],
                  f.lcs_celltot, f.lcs_tiletot, stray);
    if (nt > 0)
      EMSESG_LAUNCH(ctx, "lcs_tail_count", k_lcs_tail_count, nblk(nt), 256, 0, tk, nt, deadkey, (int)tcells,
                    f.lcs_celltot, (unsigned long long*)f.lcs_tiletot, stray);
    EMSESG_LAUNCH(ctx, "lcs_tiles", k_lcs_tiles, 1, 1024, 0, f.lcs_tiletot, f.ntiles, ts2, tp2, f.count_d + is,
                  f.slots_d + is, stray);
    EMSESG_LAUNCH(ctx, "lcs_bases", k_lcs_bases, (unsigned)f.ntiles, CELL_THREADS, 0, cnt, f.lcs_celltot, g, G[is],
                  ts2, tp2, bas, f.lcs_inv + off, stray);
    EMSESG_LAUNCH(ctx, "lcs_rank", k_lcs_rank, (unsigned)f.ntiles, PUSH_THREADS, lsm, f.pos + off,
                  f.tile_start + is * T1, f.tile_pad + is * T1, g, G[is], f.lcs_wcnt,
                  bas, ts2, tp2, f.lcs_inv + off, ctx->d_status, ctx->d_diag, stray);
    if (nt > 0)
      EMSESG_LAUNCH(ctx, "lcs_tail_inv", k_lcs_tail_inv, nblk(nt), 256, 0, tk, tv, nt, deadkey, (int)tcells,
                    f.lcs_celltot, ts2, tp2, f.lcs_inv + off, stray);
    // the move's shape from the mean rows per tile (the host's count is an
    // upper bound between synchronisations: escapes are not in it)
    if (ctx->totalp[is] + nt <= (int64_t)MOVE_SMALL_ROWS * PUSH_THREADS * f.ntiles)
      EMSESG_LAUNCH(ctx, "lcs_move", k_lcs_move<MoveSmall>, (unsigned)f.ntiles, PUSH_THREADS, move_smem<MoveSmall>(),
                    f.pos + off, f.vx + off, f.vy + off, f.vz + off, f.tile_start + is * T1, f.tile_pad + is * T1, ts2,
                    tp2, f.lcs_inv + off, f.pos2 + off, f.vx2 + off, f.vy2 + off, f.vz2 + off, stray);
    else if (ctx->totalp[is] + nt <= (int64_t)MOVE_MID_ROWS * PUSH_THREADS * f.ntiles)
      EMSESG_LAUNCH(ctx, "lcs_move", k_lcs_move<MoveMid>, (unsigned)f.ntiles, PUSH_THREADS, move_smem<MoveMid>(),
                    f.pos + off, f.vx + off, f.vy + off, f.vz + off, f.tile_start + is * T1, f.tile_pad + is * T1, ts2,
                    tp2, f.lcs_inv + off, f.pos2 + off, f.vx2 + off, f.vy2 + off, f.vz2 + off, stray);
    else
      EMSESG_LAUNCH(ctx, "lcs_move", k_lcs_move<MoveBig>, (unsigned)f.ntiles, PUSH_THREADS, move_smem<MoveBig>(),
                    f.pos + off, f.vx + off, f.vy + off, f.vz + off, f.tile_start + is * T1, f.tile_pad + is * T1, ts2,
                    tp2, f.lcs_inv + off, f.pos2 + off, f.vx2 + off, f.vy2 + off, f.vz2 + off, stray);
    if (f.capture)
      EMSESG_LAUNCH(ctx, "lcs_keep", k_lcs_keep, 4 * 148, 256, 0, stray, f.pos + off, f.vx + off, f.vy + off,
                    f.vz + off, f.tile_start + is * T1, f.tile_pad + is * T1, f.ntiles, f.pos2 + off, f.vx2 + off,
                    f.vy2 + off, f.vz2 + off, ts2, tp2, f.lcs_inv + off);
  }
  std::swap(f.pos, f.pos2);
  std::swap(f.vx, f.vx2);
  std::swap(f.vy, f.vy2);
  std::swap(f.vz, f.vz2);
  std::swap(f.tile_start, f.tile_start2);
  std::swap(f.tile_pad, f.tile_pad2);
  for (int is = 0; is < c.nspec; is++) f.ntail[is] = 0;  // merged into the regions
  *done = true;
  return EMSESG_OK;
}

extern "C" int emsesg_fx_sort(emsesg_ctx* ctx) {
  if (!ctx) return EMSESG_ERR_ARG;
  if (!ctx->fx.loaded) return set_error(ctx, EMSESG_ERR_STATE, "FP32 form not loaded (emsesg_fx_load)");
  FxState& f = ctx->fx;
  for (int is = 0; is < ctx->cfg.nspec; is++)
    if (f.pending[is]) return set_error(ctx, EMSESG_ERR_STATE, "injected particles are sorted before their first push");
  if (f.tiled) {
    bool done = false;
    int lrc = fx_local_sort(ctx, &done);
    if (lrc) return lrc;
    if (done) return EMSESG_OK;
  }
  int64_t most = 1;
  for (int is = 0; is < ctx->cfg.nspec; is++) most = std::max(most, sort_slots(ctx, is) + f.ntail[is]);
  int rc = ensure_sort_scratch(ctx, most);
  if (rc) return rc;
  Geo g = make_geo(ctx);
  uint32_t tilecells = (uint32_t)(f.tile[0] * f.tile[1] * f.tile[2]);
  uint32_t deadkey = (uint32_t)(f.ntiles * tilecells);
  int bits = 1;
  while (bits < 32 && (1ULL << bits) <= deadkey) bits++;
  for (int is = 0; is < ctx->cfg.nspec; is++) {
    int64_t n = sort_slots(ctx, is);
    int64_t off = f.base[is];
    int64_t* ts = f.tile_start + (int64_t)is * (f.ntiles + 1);
    int64_t* tp = f.tile_pad + (int64_t)is * (f.ntiles + 1);
    if (ctx->totalp[is] == 0) {
      EMSESG_CUDA(ctx, cudaMemsetAsync(ts, 0, (f.ntiles + 1) * sizeof(int64_t), ctx->stream));
      EMSESG_CUDA(ctx, cudaMemsetAsync(tp, 0, (f.ntiles + 1) * sizeof(int64_t), ctx->stream));
      EMSESG_CUDA(ctx, cudaMemsetAsync(f.count_d + is, 0, sizeof(int64_t), ctx->stream));
      EMSESG_CUDA(ctx, cudaMemsetAsync(f.slots_d + is, 0, sizeof(int64_t), ctx->stream));
      continue;
    }
    const int64_t nt = f.ntail[is];
    EMSESG_LAUNCH(ctx, "fx_keys", k_fx_keys, nblk(n + nt), 256, 0, f.pos + off, n, f.slots_d + is, f.tail0[is], nt,
                  g, deadkey, ctx->sort.keys[0], ctx->sort.vals[0]);
    n += nt;
    f.ntail[is] = 0;
    uint32_t *ko, *vo;
    if ((rc = sort_pairs(ctx, ctx->sort.keys[0], ctx->sort.vals[0], n, bits, &ko, &vo))) return rc;
    EMSESG_LAUNCH(ctx, "fx_tile_starts", k_tile_starts, nblk(n + 1), 256, 0, ko, n, tilecells, f.ntiles, ts,
                  f.count_d + is);
    EMSESG_LAUNCH(ctx, "fx_tile_pad", k_tile_pad, 1, 1024, 0, ts, f.ntiles, tp, f.slots_d + is);
    EMSESG_LAUNCH(ctx, "fx_gather", k_fx_gather_tm, (unsigned)f.ntiles, PUSH_THREADS, 0, f.pos + off, f.vx + off,
                  f.vy + off, f.vz + off, vo, ts, tp, f.pos2 + off, f.vx2 + off, f.vy2 + off, f.vz2 + off,
                  f.lcs_inv + off);
  }
  std::swap(f.pos, f.pos2);
  std::swap(f.vx, f.vx2);
  std::swap(f.vy, f.vy2);
  std::swap(f.vz, f.vz2);
  f.tiled = true;
  return EMSESG_OK;
}

namespace emsesg {
namespace {
// Live particles inside a box body (the push's end-point test, inclusive
// bounds), counted: records loaded from a caller may start inside one.
__global__ void k_fx_count_in_boxes(const float4* __restrict__ pos, int64_t n, Geo g, Bodies bd,
                                    unsigned long long* cnt) {
  const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  const float4 p = pos[m];
  const uint32_t cell = (uint32_t)__float_as_int(p.w);
  if (cell == DEAD) return;
  int c3[3];
  unpack(g, cell, c3[0], c3[1], c3[2]);
  const float f3v[3] = {p.x, p.y, p.z};
  for (int q = 0; q < bd.n; q++) {
    if (bd.kind[q] != 0) continue;
    bool in = true;
    for (int d = 0; d < 3; d++)
      in = in && c3[d] >= bd.lo[q][d] && (c3[d] < bd.hi[q][d] || (c3[d] == bd.hi[q][d] && f3v[d] == 0.0f));
    if (in) {
      atomicAdd(cnt, 1ull);
      return;
    }
  }
}
}  // namespace
}  // namespace emsesg

extern "C" int emsesg_fx_load(emsesg_ctx* ctx) {
  if (!ctx) return EMSESG_ERR_ARG;
  if (ctx->cfg.flags & EMSESG_FLAG_FP32_ONLY)
    return set_error(ctx, EMSESG_ERR_STATE, "FP32-only context: use emsesg_fx_load_plasma");
  int rc = fx_alloc(ctx);
  if (rc) return rc;
  FxState& f = ctx->fx;
  Geo g = make_geo(ctx);
  for (int is = 0; is < ctx->cfg.nspec; is++) {
    int64_t n = ctx->totalp[is];
    if (n == 0) continue;
    EMSESG_LAUNCH(ctx, "fx_from_aos", k_fx_from_aos, nblk(n), 256, 0, ctx->pbuf + ctx->seg.base[is], n, g,
                  f.pos + f.base[is], f.vx + f.base[is], f.vy + f.base[is], f.vz + f.base[is], ctx->d_status,
                  ctx->d_diag);
  }
  // particles that start inside a box body: the next push sends the tile
  // regions next to a body down its general path, whose end-point test
  // absorbs them as the reference's push does (a particle entering a box
  // always crosses a cell face, so no later step needs it)
  f.box_inside = false;
  const Bodies bd = make_bodies(ctx->cfg);
  if (bd.n > bd.ncurved) {
    unsigned long long* cnt = reinterpret_cast<unsigned long long*>(ctx->d_scratch64);
    EMSESG_CUDA(ctx, cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), ctx->stream));
    for (int is = 0; is < ctx->cfg.nspec; is++)
      if (ctx->totalp[is])
        EMSESG_LAUNCH(ctx, "fx_in_boxes", k_fx_count_in_boxes, nblk(ctx->totalp[is]), 256, 0, f.pos + f.base[is],
                      ctx->totalp[is], g, bd, cnt);
    unsigned long long inside = 0;
    EMSESG_CUDA(ctx, cudaMemcpyAsync(&inside, cnt, sizeof(inside), cudaMemcpyDeviceToHost, ctx->stream));
    EMSESG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    f.box_inside = inside > 0;
  }
  // before the first sort the regions hold the records in buffer order
  EMSESG_CUDA(ctx, cudaMemcpyAsync(f.count_d, ctx->totalp, EMSESG_ISPEC * sizeof(int64_t), cudaMemcpyHostToDevice,
                                   ctx->stream));
  EMSESG_CUDA(ctx, cudaMemcpyAsync(f.slots_d, ctx->totalp, EMSESG_ISPEC * sizeof(int64_t), cudaMemcpyHostToDevice,
                                   ctx->stream));
  f.loaded = true;
  f.tiled = false;  // buffer order: the first sort is the radix path
  f.rho_prev = false;
  rc = emsesg_fx_sort(ctx);
  if (rc) return rc;
  return emsesg_synchronize(ctx);
}

namespace emsesg {
namespace {
// Particles whose start point lies inside a body (the absorption test of
// the push: a box with inclusive bounds, a cylinder or a sphere) are not
// placed: DEAD.
__global__ void k_fx_clear_bodies(float4* pos, int64_t n, Geo g, Bodies bd) {
  const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  const float4 p = pos[m];
  const uint32_t cell = (uint32_t)__float_as_int(p.w);
  if (cell == DEAD) return;
  int c3[3];
  unpack(g, cell, c3[0], c3[1], c3[2]);
  const float f3v[3] = {p.x, p.y, p.z};
  for (int q = 0; q < bd.n; q++) {
    if (bd.kind[q] != 0) {
      if (in_curved(bd, q, c3, f3v)) {
        pos[m].w = __int_as_float((int)DEAD);
        return;
      }
      continue;
    }
    bool in = true;
    for (int d = 0; d < 3; d++)
      in = in && c3[d] >= bd.lo[q][d] && (c3[d] < bd.hi[q][d] || (c3[d] == bd.hi[q][d] && f3v[d] == 0.0f));
    if (in) {
      pos[m].w = __int_as_float((int)DEAD);
      return;
    }
  }
}
}  // namespace
}  // namespace emsesg

// The records come through a bounded device scratch in chunks and are
// converted by the same kernel as emsesg_fx_load, so the state is the one
// emsesg_load_plasma + emsesg_fx_load give (without bodies: particles that
// start inside a body are left out here).
extern "C" int emsesg_fx_load_plasma(emsesg_ctx* ctx, const emsesg_plasma* pl) {
  if (!ctx || !pl) return EMSESG_ERR_ARG;
  const emsesg_config& c = ctx->cfg;
  std::string why;
  if (!bodies_supported(c, &why)) return set_error(ctx, EMSESG_ERR_UNSUPPORTED, "%s", why.c_str());
  const int64_t ncell = (int64_t)c.nx * c.ny * c.nz;
  for (int is = 0; is < c.nspec; is++) {
    const int64_t n = ncell * pl->ppc[is];
    if (pl->ppc[is] < 0 || n > ctx->seg.capacity[is])
      return set_error(ctx, EMSESG_ERR_OVERFLOW, "species %d: %lld particles exceed capacity", is + 1, (long long)n);
  }
  int rc = fx_alloc(ctx);
  if (rc) return rc;
  FxState& f = ctx->fx;
  Geo g = make_geo(ctx);
  int64_t most = 0;
  for (int is = 0; is < c.nspec; is++) most = std::max(most, ncell * pl->ppc[is]);
  const int64_t chunk = std::min<int64_t>(std::max<int64_t>(most, 1), 1 << 25);  // 2 GiB of records at most
  emsesg_particle* tmp = nullptr;
  EMSESG_CUDA(ctx, cudaMalloc(&tmp, chunk * sizeof(emsesg_particle)));
  for (int is = 0; is < c.nspec && !rc; is++) {
    const int64_t n = ncell * pl->ppc[is];
    ctx->totalp[is] = n;
    for (int64_t m0 = 0; m0 < n && !rc; m0 += chunk) {
      const int64_t k = std::min(chunk, n - m0);
      rc = plasma_records(ctx, tmp, is, m0, k, pl);
      if (rc) break;
      const int64_t o = f.base[is] + m0;
      cudaError_t e;
      k_fx_from_aos<<<nblk(k), 256, 0, ctx->stream>>>(tmp, k, g, f.pos + o, f.vx + o, f.vy + o, f.vz + o,
                                                     ctx->d_status, ctx->d_diag);
      if ((e = cudaGetLastError()) != cudaSuccess) rc = check_cuda(ctx, e, "fx_from_aos");
    }
  }
  cudaStreamSynchronize(ctx->stream);
  cudaFree(tmp);
  if (rc) return rc;
  const Bodies bd = make_bodies(c);
  if (bd.n > 0)
    for (int is = 0; is < c.nspec; is++)
      if (ctx->totalp[is])
        EMSESG_LAUNCH(ctx, "fx_clear_bodies", k_fx_clear_bodies, nblk(ctx->totalp[is]), 256, 0, f.pos + f.base[is],
                      ctx->totalp[is], g, bd);
  EMSESG_CUDA(ctx, cudaMemcpyAsync(ctx->d_count, ctx->totalp, EMSESG_ISPEC * sizeof(int64_t), cudaMemcpyHostToDevice,
                                   ctx->stream));
  EMSESG_CUDA(ctx, cudaMemcpyAsync(f.count_d, ctx->totalp, EMSESG_ISPEC * sizeof(int64_t), cudaMemcpyHostToDevice,
                                   ctx->stream));
  EMSESG_CUDA(ctx, cudaMemcpyAsync(f.slots_d, ctx->totalp, EMSESG_ISPEC * sizeof(int64_t), cudaMemcpyHostToDevice,
                                   ctx->stream));
  f.loaded = true;
  f.tiled = false;
  f.rho_prev = false;
  f.box_inside = false;  // cleared above
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
  if (ctx->cfg.flags & EMSESG_FLAG_FP32_ONLY)
    return set_error(ctx, EMSESG_ERR_STATE, "FP32-only context: no FP64 particle records");
  // Sorted order of the last sort (tile-major cell order); particles that
  // died since then come out with nid = -1 in place, as the reference leaves
  // them before transbound.
  int rc;
  // injected particles still in the tail zone join the regions first
  for (int is = 0; is < ctx->cfg.nspec; is++)
    if (ctx->fx.ntail[is] > 0) {
      if ((rc = emsesg_fx_sort(ctx))) return rc;
      break;
    }
  int64_t cnt[EMSESG_ISPEC] = {0};
  rc = emsesg_fx_counts(ctx, cnt);
  if (rc) return rc;
  FxState& f = ctx->fx;
  Geo g = make_geo(ctx);
  for (int is = 0; is < ctx->cfg.nspec; is++) {
    int64_t off = f.base[is];
    ctx->totalp[is] = cnt[is];
    if (cnt[is] == 0) continue;
    const int64_t* ts = f.tile_start + (int64_t)is * (f.ntiles + 1);
    const int64_t* tp = f.tile_pad + (int64_t)is * (f.ntiles + 1);
    EMSESG_LAUNCH(ctx, "fx_to_aos", k_fx_to_aos_tm, (unsigned)f.ntiles, PUSH_THREADS, 0, f.pos + off, f.vx + off,
                  f.vy + off, f.vz + off, ts, tp, g, is, ctx->pbuf + ctx->seg.base[is]);
  }
  EMSESG_CUDA(ctx, cudaMemcpyAsync(ctx->d_count, ctx->totalp, EMSESG_ISPEC * sizeof(int64_t), cudaMemcpyHostToDevice,
                                   ctx->stream));
  return emsesg_synchronize(ctx);
}

namespace {
int fx_step_impl(emsesg_ctx* ctx, int ustep, int do_sort, bool deposit);
}

extern "C" int emsesg_fx_step(emsesg_ctx* ctx, int ustep, int do_sort) {
  return fx_step_impl(ctx, ustep, do_sort, true);
}

namespace emsesg {
// The parts of a push whose eb arrives in z chunks: part p takes the tile
// layers tz0 .. tz1 - 1 (tiles tile[p] .. tile[p+1] - 1) and needs the node
// planes 0..zready[p] (its tiles' boxes: tz1 - 1 times the tile edge plus
// the compiled box).  The parts grow (1/16, 3/16, 3/8 and 3/8 of the
// layers, at least one each): the first starts after a small chunk, and
// each later chunk arrives while the parts before it push.  Returns the
// number of parts, 0 where the step does not run in parts (FP32 form not
// loaded, slab mode, one tile layer).
int fx_eb_plan(const emsesg_ctx* ctx, int* zready, int64_t* tile) {
  const FxState& f = ctx->fx;
  if (!f.loaded || f.slab || f.ntile[2] < 2) return 0;
  static_assert(EMSESG_EB_PARTS == 4, "one cumulative share per part");
  constexpr double share[EMSESG_EB_PARTS] = {1.0 / 16, 4.0 / 16, 10.0 / 16, 1.0};
  const int nz = ctx->cfg.nz, ntz = f.ntile[2];
  const int parts = std::min(EMSESG_EB_PARTS, ntz);
  const int tmax = std::max(f.tile[0], std::max(f.tile[1], f.tile[2]));
  const int64_t layer = (int64_t)f.ntile[0] * f.ntile[1];
  int tz0 = 0;
  for (int p = 0; p < parts; p++) {
    // at least one layer, and one left for each later part
    int tz1 = p == parts - 1 ? ntz : (int)(ntz * share[EMSESG_EB_PARTS - parts + p] + 0.5);
    tz1 = std::min(std::max(tz1, tz0 + 1), ntz - (parts - 1 - p));
    tile[p] = tz0 * layer;
    zready[p] = p == parts - 1 ? nz : std::min(nz, (tz1 - 1) * f.tile[2] + fx_box_tile(tmax) + PG);
    tz0 = tz1;
  }
  tile[parts] = f.ntiles;
  return parts;
}
}  // namespace emsesg

namespace {
// The push of one step: grdcrt, the particles of the tile regions and of the
// tail zones, into the zeroed int64 accumulators (the J of injection
// currents kept); without `deposit` the move only (no rho / J), for
// recomputing particle states on a grid without bodies or injected
// particles.  In slab mode the particles leaving through the z faces go to
// the outbox.
int fx_push_phase(emsesg_ctx* ctx, int ustep, bool deposit, bool jd) {
  if (!ctx) return EMSESG_ERR_ARG;
  if (!ctx->fx.loaded) return set_error(ctx, EMSESG_ERR_STATE, "FP32 form not loaded (emsesg_fx_load)");
  if (ustep < 1) return set_error(ctx, EMSESG_ERR_ARG, "ustep must be >= 1");
  const emsesg_config& c = ctx->cfg;
  std::string why;
  if (!bodies_supported(c, &why)) return set_error(ctx, EMSESG_ERR_UNSUPPORTED, "%s", why.c_str());
  FxState& f = ctx->fx;
  // an eb copied in z chunks: the push runs in parts, part p once chunk p is
  // there (the plan it was copied with still holds, no graph capture)
  int zready[EMSESG_EB_PARTS];
  int64_t ptile[EMSESG_EB_PARTS + 1];
  int parts = 0;
  if (deposit && ctx->eb_next_pending && ctx->eb_parts > 1 && !f.capture) {
    parts = fx_eb_plan(ctx, zready, ptile);
    for (int p = 0; parts && p < parts; p++)
      if (zready[p] != ctx->eb_zready[p] || ptile[p + 1] != ctx->eb_tile[p + 1]) parts = 0;
    if (parts != ctx->eb_parts) parts = 0;
  }
  if (parts) {
    std::swap(ctx->field[EMSESG_FIELD_EB], ctx->eb_next);
    ctx->eb_next_pending = false;
  } else {
    int rc0 = apply_pending_eb(ctx);
    if (rc0) return rc0;
  }
  Geo g = make_geo(ctx);
  const int64_t nplane = (int64_t)(c.nx + 1) * (c.ny + 1);
  if (!parts)
    EMSESG_LAUNCH(ctx, "fx_grdcrt", k_grdcrt32, nblk(nplane * (c.nz + 1)), 256, 0, ctx->field[EMSESG_FIELD_EB],
                  f.fnode, f.fnode2, field_desc(c, EMSESG_FIELD_EB), c.nx, c.ny, 0, c.nz + 1, c.e0[0], c.e0[1],
                  c.e0[2], c.b0[0], c.b0[1], c.b0[2]);
  FieldDesc fr = field_desc(c, EMSESG_FIELD_RHO), fj = field_desc(c, EMSESG_FIELD_AJ);
  unsigned long long* acc_rho = (unsigned long long*)f.accum;
  unsigned long long* acc_j = acc_rho + fr.size();
  // rho and J start from zero; J keeps the injection currents of the
  // supervisors called since the last step (emsesg_fx_inflow_current).  A
  // step without the current (jd false) leaves J's accumulator alone.
  if (deposit) {
    const int64_t nz = fr.size() + (jd && !f.inj_j_pending ? fj.size() : 0);
    EMSESG_CUDA(ctx, cudaMemsetAsync(f.accum, 0, nz * sizeof(int64_t), ctx->stream));
    if (jd) f.inj_j_pending = false;
  }
  int tmax = std::max(f.tile[0], std::max(f.tile[1], f.tile[2]));
  int smem = fx_push_smem(tmax, !deposit || jd);
  FxPushArgs a{};
  a.pos = f.pos; a.vx = f.vx; a.vy = f.vy; a.vz = f.vz;
  a.rpos = f.pos; a.rvx = f.vx; a.rvy = f.vy; a.rvz = f.vz;
  if (!deposit && f.move_src.pos) {
    a.rpos = f.move_src.pos; a.rvx = f.move_src.vx; a.rvy = f.move_src.vy; a.rvz = f.move_src.vz;
  }
  a.tile_start = f.tile_start;
  a.tile_pad = f.tile_pad;
  a.chunk_start = f.chunk_start;
  a.ntiles = f.ntiles;
  a.chunk_rows = f.chunk_rows;
  double gustep = ustep;
  a.gustep = (float)gustep;
  a.rustep = (float)(1.0 / ustep);
  for (int is = 0; is < c.nspec; is++) {
    a.off[is] = f.base[is];
    for (int d = 0; d < 3; d++) a.npbnd[is][d] = c.npbnd[is][d];
    a.qmp[is] = (float)(c.qm[is] * gustep * 0.5);
    a.qfix[is] = (float)(c.q[is] * 1099511627776.0);
  }
  a.f0 = f.fnode; a.f1 = f.fnode2;
  a.acc_rho = acc_rho; a.acc_j = acc_j;
  a.fr = fr; a.fj = fj;
  a.g = g;
  a.nesc = ctx->d_counter->nesc;
  a.gc = ctx->d_counter;
  a.surf = f.surf;
  a.bd = make_bodies(c);
  a.status = ctx->d_status;
  a.diag = ctx->d_diag;
  a.zready = c.nz;
  a.defer = f.defer;
  if (f.slab && deposit) {
    EMSESG_CUDA(ctx, cudaMemsetAsync(f.outbox_n, 0, 2 * EMSESG_ISPEC * sizeof(unsigned long long), ctx->stream));
    a.ob = Outbox{f.outbox, f.outbox_n, f.outbox_cap};
  }
  // row chunks of the tile regions: at most ntiles + rows / chunk_rows
  int64_t rows = 0;
  for (int is = 0; is < c.nspec; is++) rows = std::max(rows, (f.cap[is] + PUSH_THREADS - 1) / PUSH_THREADS);
  EMSESG_LAUNCH(ctx, "fx_chunks", k_push_chunks, (unsigned)c.nspec, 1024, 0, f.tile_start, f.ntiles, f.chunk_start,
                f.chunk_rows);
  dim3 grid((unsigned)(f.ntiles + rows / f.chunk_rows + 1), (unsigned)c.nspec);
  if (!deposit) {
    for (int is = 0; is < c.nspec; is++)
      if (f.ntail[is]) return set_error(ctx, EMSESG_ERR_STATE, "move-only step with injected particles");
    if (a.bd.n > 0) return set_error(ctx, EMSESG_ERR_UNSUPPORTED, "move-only step with bodies");
    if (fx_box_tile(tmax) == 4)
      EMSESG_LAUNCH(ctx, "fx_move", (k_fx_push<4, false>), grid, PUSH_BLOCK, smem, a);
    else
      EMSESG_LAUNCH(ctx, "fx_move", (k_fx_push<8, false>), grid, PUSH_BLOCK, smem, a);
    return EMSESG_OK;
  }
  // tile regions next to a body take the general path when a particle can
  // end inside one without leaving its cell: always with cylinders or
  // spheres, with boxes only while loaded particles may start inside one
  const bool curv = a.bd.ncurved > 0 || f.box_inside;
  const PushKernel kern = push_kernel(fx_box_tile(tmax), curv, jd);
  if (!parts) {
    EMSESG_LAUNCH(ctx, "fx_push", kern, grid, PUSH_BLOCK, smem, a);
  } else {
    const PushKernel pkern = push_kernel(fx_box_tile(tmax), curv, jd, true);
    // part p: the node planes its chunk completes (its tiles' boxes), then
    // its tiles
    int k0 = 0;
    for (int p = 0; p < parts; p++) {
      EMSESG_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->ev_ebp[p], 0));
      const int nk = zready[p] + 1 - k0;
      if (nk > 0)
        EMSESG_LAUNCH(ctx, "fx_grdcrt", k_grdcrt32, nblk(nplane * nk), 256, 0, ctx->field[EMSESG_FIELD_EB], f.fnode,
                      f.fnode2, field_desc(c, EMSESG_FIELD_EB), c.nx, c.ny, k0, nk, c.e0[0], c.e0[1], c.e0[2],
                      c.b0[0], c.b0[1], c.b0[2]);
      k0 = std::max(k0, zready[p] + 1);
      FxPushArgs ap = a;
      ap.t_lo = ptile[p];
      ap.t_n = ptile[p + 1] - ptile[p];
      ap.zready = zready[p];
      dim3 pgrid((unsigned)(ap.t_n + rows / f.chunk_rows + 1), (unsigned)c.nspec);
      EMSESG_LAUNCH(ctx, "fx_push_part", pkern, pgrid, PUSH_BLOCK, smem, ap);
    }
    // the particles the parts left, every node plane converted
    EMSESG_LAUNCH(ctx, "fx_deferred", deferred_kernel(fx_box_tile(tmax), curv, jd), nblk(f.defer_words), 256, 0,
                  a, f.defer, f.defer_words, c.nspec);
  }
  f.box_inside = false;
  // injected particles of the tail zones (general path, global deposits)
  int64_t drawn = 0;
  for (int is = 0; is < c.nspec; is++) {
    if (f.ntail[is] == 0) continue;
    EMSESG_LAUNCH(ctx, "fx_tail", (jd ? k_fx_tail<true> : k_fx_tail<false>), nblk(f.ntail[is]), 256, 0, a, is,
                  f.tail0[is], f.ntail[is],
                  f.tailord + f.tailord_base[is], ustep, c.rng_mode == 1 ? ctx->d_randoms : nullptr, ctx->n_randoms,
                  ctx->d_rand_pos, drawn, c.rng_seed, ctx->rng_stream, ctx->d_counter->nesc + is);
    drawn += f.pending[is];
    f.pending[is] = 0;
  }
  if (drawn && c.rng_mode == 1) EMSESG_LAUNCH(ctx, "fx_rand_advance", k_add_i64, 1, 1, 0, ctx->d_rand_pos, drawn);
  if (a.bd.n > 0) EMSESG_LAUNCH(ctx, "fx_chgacm", k_fx_chgacm, 1, 32, 0, ctx->d_cfg, ctx->d_counter);
  return EMSESG_OK;
}

// The fold lists of rho and J split for slab mode: the border exchange of
// the x and y axes (run by emsesg_fx_slab_begin, before the ranks exchange
// their z border planes) and the rest (run by emsesg_fx_slab_end).  Without
// slab mode the whole lists.
void fold_lists(const emsesg_config& c, bool slab, int part, std::vector<SlabOp>* rho, std::vector<SlabOp>* j) {
  for (int kind = 0; kind < 2; kind++) {
    std::vector<SlabOp> all = fold_ops(c, kind, kind == 0 ? 1 : 3);
    std::vector<SlabOp>& out = kind == 0 ? *rho : *j;
    out.clear();
    if (!slab) {
      out = all;
      continue;
    }
    int nex = 0;  // the exchange copies come first, two per periodic axis
    for (int d = 0; d < 3; d++)
      if (c.nfbnd[d] == 0) nex += 2;
    for (int q = 0; q < (int)all.size(); q++) {
      const bool exchange = q < nex;
      if (part == 0 && exchange && all[q].axis != 2) out.push_back(all[q]);
      if (part == 1 && !exchange) out.push_back(all[q]);
    }
  }
}

// The rest of a step after its push (and, in slab mode, the exchange of the
// z border planes and the arrivals): guard folds on the exact integers,
// FP64 rho and J (J first: the conversion of rho takes the continuity
// residual of the step against the rho field of the step before, still in
// place, and this J), then the re-sort after the push (so that injected
// particles take their first, partial step before they join the tile
// regions).
int fx_fields_phase(emsesg_ctx* ctx, bool jd) {
  FxState& f = ctx->fx;
  const emsesg_config& c = ctx->cfg;
  FieldDesc fr = field_desc(c, EMSESG_FIELD_RHO), fj = field_desc(c, EMSESG_FIELD_AJ);
  unsigned long long* acc_rho = (unsigned long long*)f.accum;
  unsigned long long* acc_j = acc_rho + fr.size();
  std::vector<SlabOp> orho, oj;
  fold_lists(c, f.slab, 1, &orho, &oj);
  if (!jd) oj.clear();
  int rc;
  if ((rc = run_slab_ops2(ctx, (long long*)acc_rho, fr, orho, (long long*)acc_j, fj, oj, "fx_fold"))) return rc;
  if (jd)
    EMSESG_LAUNCH(ctx, "fx_to_double", k_fix_to_double, nblk(fj.size()), 256, 0, (const long long*)acc_j,
                  ctx->field[EMSESG_FIELD_AJ], fj.size());
  unsigned long long* cres = (unsigned long long*)(f.diag + 3 * DIAG_GRID + 3);
  EMSESG_CUDA(ctx, cudaMemsetAsync(cres, 0, 2 * sizeof(double), ctx->stream));
  EMSESG_LAUNCH(ctx, "fx_to_double", k_fix_to_rho, nblk(fr.size(), RHO_BLOCK), RHO_BLOCK, 0, (const long long*)acc_rho,
                ctx->field[EMSESG_FIELD_RHO], jd ? ctx->field[EMSESG_FIELD_AJ] : nullptr, fr, fj, c.nx, c.ny, c.nz,
                cres);
  // the continuity residual needs the step's current
  f.cont_valid = jd && f.rho_prev;
  f.rho_prev = true;
  // the step's reads of eb are over: an asynchronous upload of the next eb
  // may start (inside a stream capture the event is recorded after the
  // graph's launch instead)
  if (ctx->ev_fields && !f.capture) EMSESG_CUDA(ctx, cudaEventRecord(ctx->ev_fields, ctx->stream));
  return EMSESG_OK;
}

int fx_finish_phase(emsesg_ctx* ctx, int do_sort, bool jd) {
  int rc = fx_fields_phase(ctx, jd);
  if (rc) return rc;
  ctx->rng_stream++;
  if (do_sort && (rc = emsesg_fx_sort(ctx))) return rc;
  return EMSESG_OK;
}

// One step; without `deposit` the move only (no rho / J): for recomputing
// particle states on a grid without bodies or injected particles.
int fx_step_impl(emsesg_ctx* ctx, int ustep, int do_sort, bool deposit) {
  if (ctx && ctx->fx.slab && deposit)
    return set_error(ctx, EMSESG_ERR_STATE, "slab mode: steps are emsesg_fx_slab_begin / _arrive / _end");
  int rc = fx_push_phase(ctx, ustep, deposit, true);
  if (rc) return rc;
  if (!deposit) {
    ctx->rng_stream++;
    if (do_sort && (rc = emsesg_fx_sort(ctx))) return rc;
    return EMSESG_OK;
  }
  return fx_finish_phase(ctx, do_sort, true);
}
}  // namespace

// The electrostatic step of the FP32 form: psolve2 + charge (push, boundary
// rules and bodies, rho; no current), the folds of rho and its conversion,
// then the re-sort on a sort step.  The J accumulator and the aj field are
// left as they are.
extern "C" int emsesg_fx_step_es(emsesg_ctx* ctx, int ustep, int do_sort) {
  if (!ctx) return EMSESG_ERR_ARG;
  if (ctx->fx.slab) return set_error(ctx, EMSESG_ERR_STATE, "slab mode: the electrostatic step is not built for slabs");
  int rc = fx_push_phase(ctx, ustep, true, false);
  if (rc) return rc;
  return fx_finish_phase(ctx, do_sort, false);
}

extern "C" int emsesg_fx_step_download(emsesg_ctx* ctx, int ustep, int do_sort, double* rho, double* aj) {
  if (!ctx || !rho || !aj) return EMSESG_ERR_ARG;
  if (ctx->fx.slab) return set_error(ctx, EMSESG_ERR_STATE, "slab mode: steps are emsesg_fx_slab_begin / _arrive / _end");
  int rc = side_stream(ctx);
  if (rc) return rc;
  if ((rc = fx_push_phase(ctx, ustep, true, true))) return rc;
  if ((rc = fx_fields_phase(ctx, true))) return rc;
  // rho and aj are final: copied to the host on the side stream while the
  // context's stream goes on with the sort
  const emsesg_config& c = ctx->cfg;
  const int64_t nr = field_desc(c, EMSESG_FIELD_RHO).size(), na = field_desc(c, EMSESG_FIELD_AJ).size();
  EMSESG_CUDA(ctx, cudaStreamWaitEvent(ctx->side, ctx->ev_fields, 0));
  EMSESG_CUDA(ctx, cudaMemcpyAsync(rho, ctx->field[EMSESG_FIELD_RHO], nr * sizeof(double), cudaMemcpyDeviceToHost,
                                   ctx->side));
  EMSESG_CUDA(ctx, cudaMemcpyAsync(aj, ctx->field[EMSESG_FIELD_AJ], na * sizeof(double), cudaMemcpyDeviceToHost,
                                   ctx->side));
  ctx->rng_stream++;
  if (do_sort && (rc = emsesg_fx_sort(ctx))) return rc;
  EMSESG_CUDA(ctx, cudaStreamSynchronize(ctx->side));
  return EMSESG_OK;
}

extern "C" int emsesg_fx_em_step(emsesg_ctx* ctx, int ustep, int do_sort, double tcs) {
  if (!ctx) return EMSESG_ERR_ARG;
  const emsesg_config& c = ctx->cfg;
  for (int d = 0; d < 3; d++)
    if (c.nfbnd[d] != 0) return set_error(ctx, EMSESG_ERR_UNSUPPORTED, "field step: periodic fields only");
  if (c.npc > 0 && c.line_mode != 1)
    return set_error(ctx, EMSESG_ERR_UNSUPPORTED, "field step: no body field corrections (bdyfld)");
  int rc;
  if ((rc = emsesg_bfield(ctx, 1))) return rc;  // b(n-1/2) -> b(n)
  if ((rc = emsesg_fx_step(ctx, ustep, do_sort))) return rc;
  if ((rc = emsesg_bfield(ctx, 1))) return rc;  // b(n) -> b(n+1/2)
  if ((rc = emsesg_efield(ctx, 1, tcs, 2.0))) return rc;
  return emsesg_exchange_eb(ctx);
}

namespace emsesg {
namespace {

// Checks of an injection of n records of species index is, and room in the
// device staging buffers.
int inject_reserve(emsesg_ctx* ctx, int is, int64_t n) {
  FxState& f = ctx->fx;
  if (f.ntail[is] + n > f.tailcap[is])
    return set_error(ctx, EMSESG_ERR_OVERFLOW, "tail zone of species %d full (%lld + %lld > %lld)", is + 1,
                     (long long)f.ntail[is], (long long)n, (long long)f.tailcap[is]);
  if (ctx->totalp[is] + n > ctx->seg.capacity[is])
    return set_error(ctx, EMSESG_ERR_OVERFLOW, "species %d capacity %lld exceeded", is + 1,
                     (long long)ctx->seg.capacity[is]);
  if (n > f.stage_cap) {
    cudaFree(f.stage);
    cudaFree(f.stage_ord);
    f.stage = nullptr;
    f.stage_ord = nullptr;
    f.stage_cap = 0;
    EMSESG_CUDA(ctx, cudaMalloc(&f.stage, n * sizeof(emsesg_particle)));
    EMSESG_CUDA(ctx, cudaMalloc(&f.stage_ord, n * sizeof(int32_t)));
    f.stage_cap = n;
  }
  return EMSESG_OK;
}

// The staged records (and ordinals) into the tail zone of species is; k1 is
// the pending ordinal count after them.
int inject_staged(emsesg_ctx* ctx, int is, int64_t n, int64_t k1) {
  FxState& f = ctx->fx;
  const int64_t off = f.base[is], slot0 = f.tail0[is] + f.ntail[is];
  Bodies bd = make_bodies(ctx->cfg);
  EMSESG_LAUNCH(ctx, "fx_inject", k_fx_inject, nblk(n), 256, 0, f.stage, f.stage_ord, n, make_geo(ctx), bd, slot0,
                f.pos + off, f.vx + off, f.vy + off, f.vz + off, f.tailord + f.tailord_base[is] + f.ntail[is],
                f.surf + (int64_t)is * f.nsurf, ctx->d_status, ctx->d_diag);
  f.ntail[is] += n;
  f.pending[is] = k1;
  ctx->totalp[is] += n;
  return EMSESG_OK;
}

// The supervisors' arithmetic without fused multiply-adds, so that the
// records equal those of the host supervisors (ctca_b200/inject.py).
__device__ __forceinline__ double lin(double lo, double hi, double u) {
  return __dadd_rn(lo, __dmul_rn(__dsub_rn(hi, lo), u));
}

// Emitted pairs (psuper3.F90:142-208): pair k -> records 2k (anti-particle
// on the face) and 2k+1 (its twin 1e-5 off the face, preside 1; the
// reference adds 1e-5 as a single precision literal, so the offset is
// (double)1e-5f).
__global__ void k_gen_emit(emsesg_particle* out, int32_t* ord, int64_t n, int nemd, double grd, double b1lo,
                           double b1hi, double b2lo, double b2hi, const double* __restrict__ vnorm,
                           const double* __restrict__ vtang, int npr, uint64_t seed, uint64_t stream,
                           uint64_t index0, int spec, int64_t pending) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  double u[6];
  for (int c = 0; c < 6; c++) u[c] = hash_u01(seed, stream, (index0 + (uint64_t)k) * 6 + c);
  const int an = abs(nemd);
  const int ax0 = an - 1, ax1 = an % 3, ax2 = (an + 1) % 3;  // (0,1,2), (1,2,0), (2,0,1)
  const double ud = nemd > 0 ? 1.0 : -1.0;
  const int a0 = (int)(npr * u[0]), a1 = (int)(npr * u[1]), a2 = (int)(npr * u[2]);
  const double vn = ud * vnorm[a0], vt1 = vtang[a1], vt2 = vtang[a2];
  const double rt1 = lin(b1lo, b1hi, u[4]), rt2 = lin(b2lo, b2hi, u[5]);
  emsesg_particle p;
  double* r = &p.x;
  double* v = &p.vx;
  r[ax0] = grd; r[ax1] = rt1; r[ax2] = rt2;
  v[ax0] = vn; v[ax1] = vt1; v[ax2] = vt2;
  p.pid = 0; p.nid = 0; p.spec = spec;
  p.preside = EMSESG_PCL_TO_BE_ACCUMULATED_AS_ANTIPCL;
  out[2 * k] = p;
  ord[2 * k] = 0;
  r[ax0] = __dadd_rn(grd, __dmul_rn(ud, (double)1e-5f));
  p.preside = EMSESG_PCL_INJECTED;
  out[2 * k + 1] = p;
  ord[2 * k + 1] = (int32_t)(pending + k + 1);
}

// Particles emitted from a cylindrical body (psuper3.F90:241-528), each a
// record with preside 1 and, with `anti`, its anti-particle (preside -2) at
// the same place.  The uniforms of particle k are entries per*k + c of the
// call's flat array of 6n (per = 5 for a side of radius < 1 with omni 0,
// else 6), entry j the hash of index0*6 + j.  An end cap (|nemd| = align):
// normal ud * vnormf, tangential vtangf, the point at grd, radius *
// runiform from the axis at the angle 2 pi u4.  A side: vnormc / vtangc
// turned by psicos + psi (radius >= 1), by psi (radius < 1: the point where
// the velocity's direction meets the circle) or by 2 pi u2 (omni 1), the
// coordinate along the axis hl + (hu - hl) u.  The records match the host's
// (ctca_b200/inject.emit_cylinder) up to the last bits of the device's
// cos / sin.
struct CylTabs {
  const double *vnormf, *vtangf, *runiform, *vnormc, *vtangc, *psicos;
};
__global__ void k_gen_emit_cyl(emsesg_particle* out, int32_t* ord, int64_t n, int nemd, int align, double radius,
                               double axis0, double axis1, int omni, double grd, double hl, double hu, double psi,
                               CylTabs t, int npr, int anti, uint64_t seed, uint64_t stream, uint64_t index0,
                               int spec, int64_t pending) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const bool cap = abs(nemd) == align;
  const int per = (!cap && omni == 0 && radius < 1.0) ? 5 : 6;
  double u[6];
  for (int c = 0; c < per; c++) u[c] = hash_u01(seed, stream, index0 * 6 + (uint64_t)(per * k + c));
  int ad[4];
  for (int c = 0; c < 4; c++) ad[c] = (int)(npr * u[c]);
  const double pi2 = 6.283185307179586;  // 2 acos(-1)
  int p0, p1, p2;
  double vn, vt1, vt2, rn, rt1, rt2;
  if (cap) {
    const int an = abs(nemd);
    p0 = an - 1; p1 = an % 3; p2 = (an + 1) % 3;
    vn = nemd > 0 ? t.vnormf[ad[0]] : -t.vnormf[ad[0]];
    vt1 = t.vtangf[ad[1]];
    vt2 = t.vtangf[ad[2]];
    const double radial = __dmul_rn(radius, t.runiform[ad[3]]);
    const double ang = __dmul_rn(pi2, u[4]);
    rn = grd;
    rt1 = __dadd_rn(axis0, __dmul_rn(radial, cos(ang)));
    rt2 = __dadd_rn(axis1, __dmul_rn(radial, sin(ang)));
  } else {
    double a1 = axis0, a2 = axis1;
    if (align == 1) {
      p0 = 2; p1 = 1; p2 = 0;
      a1 = axis1; a2 = axis0;
    } else if (align == 2) {
      p0 = 2; p1 = 0; p2 = 1;
    } else {
      p0 = 0; p1 = 1; p2 = 2;
    }
    const double nc = t.vnormc[ad[0]], tc = t.vtangc[ad[1]];
    if (omni == 0 && radius >= 1.0) {
      const double ang = __dadd_rn(t.psicos[ad[2]], psi);
      const double ca = cos(ang), sa = sin(ang);
      vn = __dsub_rn(__dmul_rn(nc, ca), __dmul_rn(tc, sa));
      vt1 = __dadd_rn(__dmul_rn(nc, sa), __dmul_rn(tc, ca));
      rn = __dadd_rn(a1, __dmul_rn(radius, ca));
      rt1 = __dadd_rn(a2, __dmul_rn(radius, sa));
      vt2 = t.vtangf[ad[3]];
      rt2 = lin(hl, hu, u[5]);
    } else if (omni == 0) {
      const double ca = cos(psi), sa = sin(psi);
      vn = __dsub_rn(__dmul_rn(nc, ca), __dmul_rn(tc, sa));
      vt1 = __dadd_rn(__dmul_rn(nc, sa), __dmul_rn(tc, ca));
      vt2 = t.vtangf[ad[2]];
      const double v2normi = __ddiv_rn(radius, __dsqrt_rn(__dadd_rn(__dmul_rn(vn, vn), __dmul_rn(vt1, vt1))));
      rn = __dadd_rn(a1, __dmul_rn(vn, v2normi));
      rt1 = __dadd_rn(a2, __dmul_rn(vt1, v2normi));
      rt2 = lin(hl, hu, u[4]);
    } else {
      const double eaz = __dmul_rn(pi2, u[2]);
      const double ca = cos(eaz), sa = sin(eaz);
      vn = __dsub_rn(__dmul_rn(nc, ca), __dmul_rn(tc, sa));
      vt1 = __dadd_rn(__dmul_rn(nc, sa), __dmul_rn(tc, ca));
      vt2 = t.vtangf[ad[3]];
      rn = __dadd_rn(a1, __dmul_rn(radius, ca));
      rt1 = __dadd_rn(a2, __dmul_rn(radius, sa));
      rt2 = lin(hl, hu, u[5]);
    }
  }
  emsesg_particle p;
  double* r = &p.x;
  double* v = &p.vx;
  r[p0] = rn; r[p1] = rt1; r[p2] = rt2;
  v[p0] = vn; v[p1] = vt1; v[p2] = vt2;
  p.pid = 0; p.nid = 0; p.spec = spec;
  p.preside = EMSESG_PCL_INJECTED;
  const int64_t o = anti ? 2 * k : k;
  out[o] = p;
  ord[o] = (int32_t)(pending + k + 1);
  if (anti) {
    p.preside = EMSESG_PCL_TO_BE_ACCUMULATED_AS_ANTIPCL;
    out[o + 1] = p;
    ord[o + 1] = 0;
  }
}

// Particles emitted from a rectangular plane (psuper2.F90:330-360,
// 554-576): the normal coordinate grd + vn * injctisw * u3, the tangential
// ones uniform on the plane plus vt * injctisw * u3; preside 0, pid = the
// body.  One record per particle.
__global__ void k_gen_emit_plane(emsesg_particle* out, int32_t* ord, int64_t n, int nemd, double grd, double b1lo,
                                 double b1hi, double b2lo, double b2hi, const double* __restrict__ vnorm,
                                 const double* __restrict__ vtang, int npr, double injctisw, int pid,
                                 uint64_t seed, uint64_t stream, uint64_t index0, int spec) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  double u[6];
  for (int c = 0; c < 6; c++) u[c] = hash_u01(seed, stream, (index0 + (uint64_t)k) * 6 + c);
  const int an = abs(nemd);
  const int ax0 = an - 1, ax1 = an % 3, ax2 = (an + 1) % 3;
  const double ud = nemd > 0 ? 1.0 : -1.0;
  const int a0 = (int)(npr * u[0]), a1 = (int)(npr * u[1]), a2 = (int)(npr * u[2]);
  const double vn = ud * vnorm[a0], vt1 = vtang[a1], vt2 = vtang[a2];
  emsesg_particle p;
  double* r = &p.x;
  double* v = &p.vx;
  r[ax0] = __dadd_rn(grd, __dmul_rn(__dmul_rn(vn, injctisw), u[3]));
  r[ax1] = __dadd_rn(lin(b1lo, b1hi, u[4]), __dmul_rn(__dmul_rn(vt1, injctisw), u[3]));
  r[ax2] = __dadd_rn(lin(b2lo, b2hi, u[5]), __dmul_rn(__dmul_rn(vt2, injctisw), u[3]));
  v[ax0] = vn; v[ax1] = vt1; v[ax2] = vt2;
  p.pid = pid; p.preside = 0; p.nid = 0; p.spec = spec;
  out[k] = p;
  ord[k] = 0;
}

// Inflow through the lower (front) or upper face of `axis`
// (psuper2.F90:114-292): u2, u3, u4 give x, y, z -- uniform on the face
// along the tangential axes; along the normal the distance vn * injctisw * u
// from the face.  vnt: normal speeds [int(npr*u0)]; vat / vbt: the
// tangential ones of the two other axes in increasing order [int(npr*u1)].
// The injection current of psuper1 (psuper1.F90:120-323 with
// current_deposition, :859-988) for a particle injected through the face
// (axis, front) at a: the zigzag current of the path from b outside the face
// (-1 below the lower face, n + 0.99999999 above the upper one, along the
// normal; a - v ustep along the others) to a, times q, into the int64 J
// accumulator (scale 2^40), each of the 24 contributions rounded on its own.
// A node outside the accumulator's guard layers is reported, not written.
struct InjCurrent {
  long long* acc;  // J accumulator; null: no current
  FieldDesc fj;
  double qfix;     // q * 2^40
  int ustep;
  double rustep;
};

__device__ __forceinline__ void inj_zigzag(const InjCurrent& c, const double (&b)[3], const double (&a)[3], int* status,
                                           long long* diag) {
  int ib[3], ia[3];
  double r[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    ib[d] = (int)floor(b[d]);
    ia[d] = (int)floor(a[d]);
    r[d] = ib[d] == ia[d] ? __dmul_rn(__dadd_rn(b[d], a[d]), 0.5) : fmax((double)ib[d], (double)ia[d]);
  }
  const int ext[3] = {c.fj.ex, c.fj.ey, c.fj.ez};
#pragma unroll
  for (int s = 0; s < 2; s++) {
    double dd[3], vv[3];
    int cell[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      if (s == 0) {
        cell[d] = ib[d];
        dd[d] = __dsub_rn(__dmul_rn(__dadd_rn(r[d], b[d]), 0.5), (double)ib[d]);
        vv[d] = __dmul_rn(__dsub_rn(r[d], b[d]), c.rustep);
      } else {
        cell[d] = ia[d];
        dd[d] = __dsub_rn(__dmul_rn(__dadd_rn(a[d], r[d]), 0.5), (double)ia[d]);
        vv[d] = __dmul_rn(__dsub_rn(a[d], r[d]), c.rustep);
      }
    }
#pragma unroll
    for (int comp = 0; comp < 3; comp++) {
      const int e1 = comp == 0 ? 1 : 0, e2 = comp == 2 ? 1 : 2;
      const double w4 = __dmul_rn(dd[e1], dd[e2]);
      const double w[4] = {__dsub_rn(__dsub_rn(1.0, dd[e1]), __dsub_rn(dd[e2], w4)), __dsub_rn(dd[e1], w4),
                           __dsub_rn(dd[e2], w4), w4};
#pragma unroll
      for (int q = 0; q < 4; q++) {
        int n3[3] = {cell[0], cell[1], cell[2]};
        if (q & 1) n3[e1]++;
        if (q & 2) n3[e2]++;
        bool in = true;
#pragma unroll
        for (int d = 0; d < 3; d++) in = in && n3[d] >= c.fj.lo && n3[d] - c.fj.lo < ext[d];
        if (!in) {
          report_bad(status, diag, SITE_FX_DEPOSIT, -5, n3[0] + 100000LL * n3[1] + 10000000000LL * n3[2]);
          continue;
        }
        const long long v = __double2ll_rn(__dmul_rn(__dmul_rn(vv[comp], w[q]), c.qfix));
        if (v) atomicAdd((unsigned long long*)&c.acc[c.fj.at(comp, n3[0], n3[1], n3[2])], (unsigned long long)v);
      }
    }
  }
}

__global__ void k_gen_inflow(emsesg_particle* out, int32_t* ord, int64_t n, int axis, int front, int nx, int ny,
                             int nz, const double* __restrict__ vnt, const double* __restrict__ vat,
                             const double* __restrict__ vbt, int npr, double injctisw, uint64_t seed,
                             uint64_t stream, uint64_t index0, int spec, InjCurrent cur, int* status,
                             long long* diag) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  double u[5];
  for (int c = 0; c < 5; c++) u[c] = hash_u01(seed, stream, (index0 + (uint64_t)k) * 5 + c);
  const int a1 = (int)(npr * u[0]), a2 = (int)(npr * u[1]);
  const int ext[3] = {nx, ny, nz};
  double x[3], v[3];
  for (int d = 0; d < 3; d++) x[d] = __dadd_rn(0.0, __dmul_rn((double)ext[d], u[2 + d]));
  const double vn = vnt[a1];
  const double dn = __dmul_rn(__dmul_rn(vn, injctisw), u[2 + axis]);
  x[axis] = front ? dn : __dadd_rn((double)ext[axis], dn);
  v[axis] = vn;
  v[axis == 0 ? 1 : 0] = vat[a2];
  v[axis == 2 ? 1 : 2] = vbt[a2];
  emsesg_particle p;
  p.x = x[0]; p.y = x[1]; p.z = x[2];
  p.vx = v[0]; p.vy = v[1]; p.vz = v[2];
  p.pid = 0; p.preside = 0; p.nid = 0; p.spec = spec;
  out[k] = p;
  ord[k] = 0;
  if (cur.acc) {
    // the point outside the face, component by component (no array index
    // chosen at run time)
    const double us = (double)cur.ustep;
    const double out_n = front ? -1.0 : __dadd_rn((double)ext[axis], 0.99999999);
    const double b[3] = {axis == 0 ? out_n : __dsub_rn(p.x, __dmul_rn(p.vx, us)),
                         axis == 1 ? out_n : __dsub_rn(p.y, __dmul_rn(p.vy, us)),
                         axis == 2 ? out_n : __dsub_rn(p.z, __dmul_rn(p.vz, us))};
    const double at[3] = {p.x, p.y, p.z};
    inj_zigzag(cur, b, at, status, diag);
  }
}

int inject_tables(emsesg_ctx* ctx, int ntab, int npr, const double* const* tabs) {
  FxState& f = ctx->fx;
  const int64_t need = (int64_t)ntab * npr;
  if (need > f.inj_tab_cap) {
    EMSESG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    cudaFree(f.inj_tab);
    f.inj_tab = nullptr;
    f.inj_tab_cap = 0;
    EMSESG_CUDA(ctx, cudaMalloc(&f.inj_tab, need * sizeof(double)));
    f.inj_tab_cap = need;
  }
  for (int t = 0; t < ntab; t++)
    EMSESG_CUDA(ctx, cudaMemcpyAsync(f.inj_tab + (int64_t)t * npr, tabs[t], npr * sizeof(double),
                                     cudaMemcpyHostToDevice, ctx->stream));
  return EMSESG_OK;
}

int inject_check(emsesg_ctx* ctx, int spec, int64_t n, int npr, const void* t0, const void* t1, const void* t2) {
  if (!ctx || n < 0 || npr < 1 || !t0 || !t1 || !t2) return EMSESG_ERR_ARG;
  if (!ctx->fx.loaded) return set_error(ctx, EMSESG_ERR_STATE, "FP32 form not loaded (emsesg_fx_load)");
  if (spec < 1 || spec > ctx->cfg.nspec) return set_error(ctx, EMSESG_ERR_ARG, "species %d out of range", spec);
  return EMSESG_OK;
}

}  // namespace
}  // namespace emsesg

namespace emsesg {
namespace {
// The charge of particles that arrived from a neighbouring slab (tail slots
// s0 .. s0 + n - 1 of a species region): the CIC weights of the push
// (charge.F90:152-210) at their FP32 offsets, into the int64 rho.
__global__ void k_fx_rho_arrivals(const float4* __restrict__ pos, int64_t s0, int64_t n, Sink sk, Geo g,
                                  float qfix) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const float4 ps = pos[s0 + k];
  const uint32_t cell = (uint32_t)__float_as_int(ps.w);
  if (cell == DEAD) return;
  int i, j, kk;
  unpack(g, cell, i, j, kk);
  const float X = ps.x, Y = ps.y, Z = ps.z;
  const float XY = X * Y, XZ = X * Z, YZ = Y * Z, Z2 = 1.0f - Z, XZ2 = X * Z2, YZ2 = Y * Z2;
  V8 R;
  R.v[2] = XY * Z; R.v[1] = XZ - R.v[2]; R.v[3] = YZ - R.v[2]; R.v[0] = Z - XZ - R.v[3];
  R.v[6] = XY * Z2; R.v[5] = XZ2 - R.v[6]; R.v[7] = YZ2 - R.v[6]; R.v[4] = Z2 - XZ2 - R.v[7];
  put_r_global(sk, i, j, kk, R, qfix);
}

// keys = source slot (pid), vals = record index, of one outbox region.
__global__ void k_outbox_keys(const emsesg_particle* __restrict__ rec, int64_t n, uint32_t* keys, uint32_t* vals) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  keys[k] = (uint32_t)rec[k].pid;
  vals[k] = (uint32_t)k;
}

__global__ void k_outbox_gather(const emsesg_particle* __restrict__ rec, const uint32_t* __restrict__ idx, int64_t n,
                                emsesg_particle* out) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  out[k] = rec[idx[k]];
}

// The z border planes of rho (kind 0) and J (kind 1) that slab mode
// exchanges, as the border exchange of oh3_exchange_borders for the types of
// src/wrapper/ohinit.F90:113-118 (rho: from 0 / to n+1 and from n / to -1,
// one plane each way; J: from -1..1 / to n+2..n+4 and from n-1..n+1 /
// to -4..-2): which 0 the planes sent down, 1 sent up, 2 received from
// below, 3 received from above.
void slab_plane_range(int kind, int which, int nz, int* k0, int* depth) {
  const int fromL = kind == 0 ? 0 : -1, toL = kind == 0 ? 1 : 2, sizeL = kind == 0 ? 1 : 3;
  const int fromU = kind == 0 ? 0 : -1, toU = kind == 0 ? -1 : -4, sizeU = kind == 0 ? 1 : 3;
  if (which == 0) { *k0 = fromL; *depth = sizeL; }
  else if (which == 1) { *k0 = nz + fromU; *depth = sizeU; }
  else if (which == 2) { *k0 = toU; *depth = sizeU; }
  else { *k0 = nz + toL; *depth = sizeL; }
}
}  // namespace
}  // namespace emsesg

extern "C" int emsesg_fx_chunk_rows(emsesg_ctx* ctx, int rows) {
  if (!ctx || rows < 1 || rows > 1 << 20) return EMSESG_ERR_ARG;
  FxState& f = ctx->fx;
  if (f.slab_open) return set_error(ctx, EMSESG_ERR_STATE, "slab step open");
  if (f.chunk_rows != rows && f.gexec) {  // a captured block holds the old grid
    cudaGraphExecDestroy(f.gexec);
    f.gexec = nullptr;
  }
  f.chunk_rows = rows;
  return EMSESG_OK;
}

extern "C" int emsesg_fx_slab(emsesg_ctx* ctx, int on, int64_t outbox_cap) {
  if (!ctx || (on && outbox_cap < 1)) return EMSESG_ERR_ARG;
  FxState& f = ctx->fx;
  if (!f.loaded) return set_error(ctx, EMSESG_ERR_STATE, "FP32 form not loaded (emsesg_fx_load)");
  if (f.slab_open) return set_error(ctx, EMSESG_ERR_STATE, "slab step open (emsesg_fx_slab_end first)");
  const emsesg_config& c = ctx->cfg;
  cudaFree(f.outbox); cudaFree(f.outbox2); cudaFree(f.outbox_n);
  f.outbox = f.outbox2 = nullptr;
  f.outbox_n = nullptr;
  f.outbox_cap = 0;
  f.slab = false;
  if (!on) return EMSESG_OK;
  for (int is = 0; is < c.nspec; is++)
    if (c.npbnd[is][2] != 0) return set_error(ctx, EMSESG_ERR_UNSUPPORTED, "slab mode: periodic z particles only");
  if (c.nfbnd[2] != 0) return set_error(ctx, EMSESG_ERR_UNSUPPORTED, "slab mode: periodic z fields only");
  if (c.npc > 0 && c.line_mode != 1) return set_error(ctx, EMSESG_ERR_UNSUPPORTED, "slab mode: no bodies");
  EMSESG_CUDA(ctx, cudaMalloc(&f.outbox, (size_t)2 * c.nspec * outbox_cap * sizeof(emsesg_particle)));
  EMSESG_CUDA(ctx, cudaMalloc(&f.outbox2, (size_t)outbox_cap * sizeof(emsesg_particle)));
  EMSESG_CUDA(ctx, cudaMalloc(&f.outbox_n, 2 * EMSESG_ISPEC * sizeof(unsigned long long)));
  f.outbox_cap = outbox_cap;
  f.slab = true;
  return EMSESG_OK;
}

extern "C" int emsesg_fx_slab_begin(emsesg_ctx* ctx, int ustep, int64_t* counts) {
  if (!ctx || !counts) return EMSESG_ERR_ARG;
  FxState& f = ctx->fx;
  if (!f.slab) return set_error(ctx, EMSESG_ERR_STATE, "not in slab mode (emsesg_fx_slab)");
  if (f.slab_open) return set_error(ctx, EMSESG_ERR_STATE, "slab step already open");
  const emsesg_config& c = ctx->cfg;
  int rc = fx_push_phase(ctx, ustep, true, true);
  if (rc) return rc;
  unsigned long long n[2 * EMSESG_ISPEC];
  EMSESG_CUDA(ctx, cudaMemcpyAsync(n, f.outbox_n, sizeof(n), cudaMemcpyDeviceToHost, ctx->stream));
  EMSESG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (int q = 0; q < 2 * c.nspec; q++)
    if ((int64_t)n[q] > f.outbox_cap)
      return set_error(ctx, EMSESG_ERR_OVERFLOW, "slab outbox %d: %llu particles left, room for %lld", q,
                       (unsigned long long)n[q], (long long)f.outbox_cap);
  // each region in the order of the particles' slots (the atomics of the
  // push leave it in any order)
  int64_t slots = 1;
  for (int is = 0; is < c.nspec; is++) slots = std::max(slots, f.base[is] + f.cap[is]);
  int bits = 1;
  while (bits < 32 && (1LL << bits) < slots) bits++;
  for (int q = 0; q < 2 * c.nspec; q++) {
    counts[q] = (int64_t)n[q];
    if (n[q] < 2) continue;
    emsesg_particle* reg = f.outbox + (int64_t)q * f.outbox_cap;
    if ((rc = ensure_sort_scratch(ctx, (int64_t)n[q]))) return rc;
    EMSESG_LAUNCH(ctx, "slab_keys", k_outbox_keys, nblk((int64_t)n[q]), 256, 0, reg, (int64_t)n[q],
                  ctx->sort.keys[0], ctx->sort.vals[0]);
    uint32_t *ko, *vo;
    if ((rc = sort_pairs(ctx, ctx->sort.keys[0], ctx->sort.vals[0], (int64_t)n[q], bits, &ko, &vo))) return rc;
    EMSESG_LAUNCH(ctx, "slab_gather", k_outbox_gather, nblk((int64_t)n[q]), 256, 0, reg, vo, (int64_t)n[q],
                  f.outbox2);
    EMSESG_CUDA(ctx, cudaMemcpyAsync(reg, f.outbox2, n[q] * sizeof(emsesg_particle), cudaMemcpyDeviceToDevice,
                                     ctx->stream));
  }
  EMSESG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  f.slab_open = true;
  return EMSESG_OK;
}

extern "C" int emsesg_fx_slab_outbox(emsesg_ctx* ctx, int spec, int dir, emsesg_particle** dev) {
  if (!ctx || !dev || dir < 0 || dir > 1) return EMSESG_ERR_ARG;
  FxState& f = ctx->fx;
  if (!f.slab) return set_error(ctx, EMSESG_ERR_STATE, "not in slab mode (emsesg_fx_slab)");
  if (spec < 1 || spec > ctx->cfg.nspec) return set_error(ctx, EMSESG_ERR_ARG, "species %d out of range", spec);
  *dev = f.outbox + (int64_t)(2 * (spec - 1) + dir) * f.outbox_cap;
  return EMSESG_OK;
}

extern "C" int emsesg_fx_slab_planes(emsesg_ctx* ctx, int which, int64_t** rho, int64_t* nrho, int64_t** j,
                                     int64_t* nj) {
  if (!ctx || !rho || !nrho || !j || !nj || which < 0 || which > 3) return EMSESG_ERR_ARG;
  FxState& f = ctx->fx;
  if (!f.slab) return set_error(ctx, EMSESG_ERR_STATE, "not in slab mode (emsesg_fx_slab)");
  const emsesg_config& c = ctx->cfg;
  FieldDesc fr = field_desc(c, EMSESG_FIELD_RHO), fj = field_desc(c, EMSESG_FIELD_AJ);
  int k0, depth;
  slab_plane_range(0, which, c.nz, &k0, &depth);
  *rho = f.accum + fr.at(0, fr.lo, fr.lo, k0);
  *nrho = (int64_t)depth * fr.nc * fr.ex * fr.ey;
  slab_plane_range(1, which, c.nz, &k0, &depth);
  *j = f.accum + fr.size() + fj.at(0, fj.lo, fj.lo, k0);
  *nj = (int64_t)depth * fj.nc * fj.ex * fj.ey;
  return EMSESG_OK;
}

extern "C" int emsesg_fx_slab_arrive(emsesg_ctx* ctx, int spec, const emsesg_particle* dev, int64_t n) {
  if (!ctx || n < 0 || (n > 0 && !dev)) return EMSESG_ERR_ARG;
  FxState& f = ctx->fx;
  if (!f.slab_open) return set_error(ctx, EMSESG_ERR_STATE, "no slab step open (emsesg_fx_slab_begin)");
  const int is = spec - 1;
  if (is < 0 || is >= ctx->cfg.nspec) return set_error(ctx, EMSESG_ERR_ARG, "species %d out of range", spec);
  if (n == 0) return EMSESG_OK;
  int rc = inject_reserve(ctx, is, n);
  if (rc) return rc;
  EMSESG_CUDA(ctx, cudaMemcpyAsync(f.stage, dev, n * sizeof(emsesg_particle), cudaMemcpyDeviceToDevice, ctx->stream));
  EMSESG_CUDA(ctx, cudaMemsetAsync(f.stage_ord, 0, n * sizeof(int32_t), ctx->stream));
  const int64_t s0 = f.base[is] + f.tail0[is] + f.ntail[is];
  if ((rc = inject_staged(ctx, is, n, f.pending[is]))) return rc;
  const emsesg_config& c = ctx->cfg;
  FieldDesc fr = field_desc(c, EMSESG_FIELD_RHO), fj = field_desc(c, EMSESG_FIELD_AJ);
  unsigned long long* acc_rho = (unsigned long long*)f.accum;
  const Sink sk{acc_rho, acc_rho + fr.size(), fr, fj, c.nx, c.ny, c.nz, ctx->d_status, ctx->d_diag};
  EMSESG_LAUNCH(ctx, "slab_rho_arrivals", k_fx_rho_arrivals, nblk(n), 256, 0, f.pos, s0, n, sk, make_geo(ctx),
                (float)(c.q[is] * 1099511627776.0));
  return EMSESG_OK;
}

extern "C" int emsesg_fx_slab_border(emsesg_ctx* ctx) {
  if (!ctx) return EMSESG_ERR_ARG;
  FxState& f = ctx->fx;
  if (!f.slab_open) return set_error(ctx, EMSESG_ERR_STATE, "no slab step open (emsesg_fx_slab_begin)");
  const emsesg_config& c = ctx->cfg;
  FieldDesc fr = field_desc(c, EMSESG_FIELD_RHO), fj = field_desc(c, EMSESG_FIELD_AJ);
  unsigned long long* acc_rho = (unsigned long long*)f.accum;
  std::vector<SlabOp> orho, oj;
  fold_lists(c, true, 0, &orho, &oj);
  int rc = run_slab_ops2(ctx, (long long*)acc_rho, fr, orho, (long long*)(acc_rho + fr.size()), fj, oj, "fx_fold");
  if (rc) return rc;
  return emsesg_synchronize(ctx);
}

extern "C" int emsesg_fx_slab_end(emsesg_ctx* ctx, int do_sort) {
  if (!ctx) return EMSESG_ERR_ARG;
  FxState& f = ctx->fx;
  if (!f.slab_open) return set_error(ctx, EMSESG_ERR_STATE, "no slab step open (emsesg_fx_slab_begin)");
  f.slab_open = false;
  return fx_finish_phase(ctx, do_sort, true);
}

extern "C" int emsesg_fx_inject(emsesg_ctx* ctx, int spec, const emsesg_particle* host, int64_t n) {
  if (!ctx || n < 0 || (n > 0 && !host)) return EMSESG_ERR_ARG;
  if (!ctx->fx.loaded) return set_error(ctx, EMSESG_ERR_STATE, "FP32 form not loaded (emsesg_fx_load)");
  const int is = spec - 1;
  if (is < 0 || is >= ctx->cfg.nspec) return set_error(ctx, EMSESG_ERR_ARG, "species %d out of range", spec);
  if (n == 0) return EMSESG_OK;
  FxState& f = ctx->fx;
  int rc = inject_reserve(ctx, is, n);
  if (rc) return rc;
  // ordinal of each injected particle's random step, in buffer order, staged
  // in pinned host memory that the previous call's upload has released
  if (!f.ord_ev) EMSESG_CUDA(ctx, cudaEventCreateWithFlags(&f.ord_ev, cudaEventDisableTiming));
  EMSESG_CUDA(ctx, cudaEventSynchronize(f.ord_ev));
  if (n > f.ord_host_cap) {
    cudaFreeHost(f.ord_host);
    f.ord_host = nullptr;
    f.ord_host_cap = 0;
    EMSESG_CUDA(ctx, cudaHostAlloc((void**)&f.ord_host, n * sizeof(int32_t), cudaHostAllocDefault));
    f.ord_host_cap = n;
  }
  int32_t* ord = f.ord_host;
  int64_t k1 = f.pending[is];
  for (int64_t k = 0; k < n; k++)
    ord[k] = (host[k].preside == EMSESG_PCL_INJECTED && host[k].nid != -1) ? (int32_t)(++k1) : 0;
  // records from pinned host memory go asynchronously; from pageable memory
  // the copy returns once the records are staged
  EMSESG_CUDA(ctx, cudaMemcpyAsync(f.stage, host, n * sizeof(emsesg_particle), cudaMemcpyHostToDevice, ctx->stream));
  EMSESG_CUDA(ctx, cudaMemcpyAsync(f.stage_ord, ord, n * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream));
  EMSESG_CUDA(ctx, cudaEventRecord(f.ord_ev, ctx->stream));
  return inject_staged(ctx, is, n, k1);
}

extern "C" int emsesg_fx_emit(emsesg_ctx* ctx, int spec, int nemd, double grd, const double* b1, const double* b2,
                              int64_t n, const double* vnorm, const double* vtang, int npr, uint64_t seed,
                              uint64_t stream, uint64_t index0) {
  int rc = inject_check(ctx, spec, n, npr, vnorm, vtang, vnorm);
  if (rc) return rc;
  if (!b1 || !b2 || nemd == 0 || nemd < -3 || nemd > 3) return set_error(ctx, EMSESG_ERR_ARG, "bad emission face");
  if (n == 0) return EMSESG_OK;
  const int is = spec - 1;
  FxState& f = ctx->fx;
  if ((rc = inject_reserve(ctx, is, 2 * n))) return rc;
  const double* tabs[2] = {vnorm, vtang};
  if ((rc = inject_tables(ctx, 2, npr, tabs))) return rc;
  const int64_t pending = f.pending[is];
  EMSESG_LAUNCH(ctx, "fx_gen_emit", k_gen_emit, nblk(n), 256, 0, f.stage, f.stage_ord, n, nemd, grd, b1[0], b1[1],
                b2[0], b2[1], f.inj_tab, f.inj_tab + npr, npr, seed, stream, index0, spec, pending);
  return inject_staged(ctx, is, 2 * n, pending + n);
}

extern "C" int emsesg_fx_emit_plane(emsesg_ctx* ctx, int spec, int nemd, double grd, const double* b1,
                                    const double* b2, int64_t n, const double* vnorm, const double* vtang, int npr,
                                    double injctisw, int pid, uint64_t seed, uint64_t stream, uint64_t index0) {
  int rc = inject_check(ctx, spec, n, npr, vnorm, vtang, vnorm);
  if (rc) return rc;
  if (!b1 || !b2 || nemd == 0 || nemd < -3 || nemd > 3) return set_error(ctx, EMSESG_ERR_ARG, "bad emission face");
  if (n == 0) return EMSESG_OK;
  const int is = spec - 1;
  FxState& f = ctx->fx;
  if ((rc = inject_reserve(ctx, is, n))) return rc;
  const double* tabs[2] = {vnorm, vtang};
  if ((rc = inject_tables(ctx, 2, npr, tabs))) return rc;
  EMSESG_LAUNCH(ctx, "fx_gen_emit_plane", k_gen_emit_plane, nblk(n), 256, 0, f.stage, f.stage_ord, n, nemd, grd,
                b1[0], b1[1], b2[0], b2[1], f.inj_tab, f.inj_tab + npr, npr, injctisw, pid, seed, stream, index0,
                spec);
  return inject_staged(ctx, is, n, f.pending[is]);
}

extern "C" int emsesg_fx_emit_cylinder(emsesg_ctx* ctx, int spec, int nemd, int align, double radius,
                                       const double* axis, int omni, double grd, double hl, double hu, double psi,
                                       int64_t n, const double* vnormf, const double* vtangf, const double* runiform,
                                       const double* vnormc, const double* vtangc, const double* psicos, int npr,
                                       int anti, uint64_t seed, uint64_t stream, uint64_t index0) {
  int rc = inject_check(ctx, spec, n, npr, vnormf, vtangf, runiform);
  if (rc) return rc;
  if (!axis || !vnormc || !vtangc || !psicos) return EMSESG_ERR_ARG;
  if (nemd == 0 || nemd < -3 || nemd > 3 || align < 1 || align > 3 || !(radius > 0.0) || (omni != 0 && omni != 1))
    return set_error(ctx, EMSESG_ERR_ARG, "bad cylinder emission (nemd %d, align %d, omni %d)", nemd, align, omni);
  if (n == 0) return EMSESG_OK;
  const int is = spec - 1;
  FxState& f = ctx->fx;
  const int64_t nrec = anti ? 2 * n : n;
  if ((rc = inject_reserve(ctx, is, nrec))) return rc;
  const double* tabs[6] = {vnormf, vtangf, runiform, vnormc, vtangc, psicos};
  if ((rc = inject_tables(ctx, 6, npr, tabs))) return rc;
  CylTabs t{f.inj_tab, f.inj_tab + npr, f.inj_tab + 2 * npr, f.inj_tab + 3 * npr, f.inj_tab + 4 * npr,
            f.inj_tab + 5 * npr};
  const int64_t pending = f.pending[is];
  EMSESG_LAUNCH(ctx, "fx_gen_emit_cyl", k_gen_emit_cyl, nblk(n), 256, 0, f.stage, f.stage_ord, n, nemd, align, radius,
                axis[0], axis[1], omni, grd, hl, hu, psi, t, npr, anti ? 1 : 0, seed, stream, index0, spec, pending);
  return inject_staged(ctx, is, nrec, pending + n);
}

namespace {
int inflow_impl(emsesg_ctx* ctx, int spec, int axis, int front, int64_t n, const double* vn_t, const double* va_t,
                const double* vb_t, int npr, double injctisw, uint64_t seed, uint64_t stream, uint64_t index0,
                int ustep) {
  int rc = inject_check(ctx, spec, n, npr, vn_t, va_t, vb_t);
  if (rc) return rc;
  if (axis < 0 || axis > 2) return set_error(ctx, EMSESG_ERR_ARG, "inflow axis %d (0, 1 or 2)", axis);
  if (ustep < 0) return set_error(ctx, EMSESG_ERR_ARG, "ustep must be >= 1");
  if (n == 0) return EMSESG_OK;
  const int is = spec - 1;
  FxState& f = ctx->fx;
  if ((rc = inject_reserve(ctx, is, n))) return rc;
  const double* tabs[3] = {vn_t, va_t, vb_t};
  if ((rc = inject_tables(ctx, 3, npr, tabs))) return rc;
  const emsesg_config& c = ctx->cfg;
  InjCurrent cur{};
  if (ustep > 0) {
    // the J accumulator: cleared before the first current after a step,
    // then kept by that step
    FieldDesc fr = field_desc(c, EMSESG_FIELD_RHO);
    cur.fj = field_desc(c, EMSESG_FIELD_AJ);
    cur.acc = (long long*)f.accum + fr.size();
    if (!f.inj_j_pending) {
      EMSESG_CUDA(ctx, cudaMemsetAsync(cur.acc, 0, cur.fj.size() * sizeof(int64_t), ctx->stream));
      f.inj_j_pending = true;
    }
    cur.qfix = c.q[is] * 1099511627776.0;
    cur.ustep = ustep;
    cur.rustep = 1.0 / ustep;
  }
  EMSESG_LAUNCH(ctx, "fx_gen_inflow", k_gen_inflow, nblk(n), 256, 0, f.stage, f.stage_ord, n, axis, front, c.nx,
                c.ny, c.nz, f.inj_tab, f.inj_tab + npr, f.inj_tab + 2 * npr, npr, injctisw, seed, stream, index0,
                spec, cur, ctx->d_status, ctx->d_diag);
  return inject_staged(ctx, is, n, f.pending[is]);
}
}  // namespace

extern "C" int emsesg_fx_inflow(emsesg_ctx* ctx, int spec, int axis, int front, int64_t n, const double* vn_t,
                                const double* va_t, const double* vb_t, int npr, double injctisw, uint64_t seed,
                                uint64_t stream, uint64_t index0) {
  return inflow_impl(ctx, spec, axis, front, n, vn_t, va_t, vb_t, npr, injctisw, seed, stream, index0, 0);
}

extern "C" int emsesg_fx_inflow_current(emsesg_ctx* ctx, int spec, int axis, int front, int64_t n,
                                        const double* vn_t, const double* va_t, const double* vb_t, int npr,
                                        double injctisw, int ustep, uint64_t seed, uint64_t stream,
                                        uint64_t index0) {
  if (ustep < 1) return ctx ? set_error(ctx, EMSESG_ERR_ARG, "ustep must be >= 1") : EMSESG_ERR_ARG;
  return inflow_impl(ctx, spec, axis, front, n, vn_t, va_t, vb_t, npr, injctisw, seed, stream, index0, ustep);
}

extern "C" int emsesg_fx_inflow_z(emsesg_ctx* ctx, int spec, int front, int64_t n, const double* vz_t,
                                  const double* vx_t, const double* vy_t, int npr, double injctisw, uint64_t seed,
                                  uint64_t stream, uint64_t index0) {
  return emsesg_fx_inflow(ctx, spec, 2, front, n, vz_t, vx_t, vy_t, npr, injctisw, seed, stream, index0);
}

extern "C" int emsesg_fx_surface(emsesg_ctx* ctx, int64_t* counts, int64_t* nsurf) {
  if (!ctx || !nsurf) return EMSESG_ERR_ARG;
  if (!ctx->fx.loaded) return set_error(ctx, EMSESG_ERR_STATE, "FP32 form not loaded");
  *nsurf = ctx->fx.nsurf;
  if (counts && ctx->fx.nsurf > 0) {
    EMSESG_CUDA(ctx, cudaMemcpyAsync(counts, ctx->fx.surf, ctx->cfg.nspec * ctx->fx.nsurf * sizeof(int64_t),
                                     cudaMemcpyDeviceToHost, ctx->stream));
    EMSESG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return EMSESG_OK;
}

extern "C" int emsesg_fx_energy(emsesg_ctx* ctx, double* engk) {
  if (!ctx || !engk) return EMSESG_ERR_ARG;
  if (!ctx->fx.loaded) return set_error(ctx, EMSESG_ERR_STATE, "FP32 form not loaded");
  FxState& f = ctx->fx;
  const emsesg_config& c = ctx->cfg;
  double* part = f.diag;
  double* sum = f.diag + 3 * DIAG_GRID;
  const double vol = (double)c.nx * (double)c.ny * (double)c.nz;
  for (int is = 0; is < c.nspec; is++) {
    const int64_t off = f.base[is];
    const int64_t* tile_end = f.tile_pad + (int64_t)is * (f.ntiles + 1) + f.ntiles;
    EMSESG_LAUNCH(ctx, "fx_energy", k_fx_energy_part, DIAG_GRID, DIAG_BLOCK, 0, f.pos + off, f.vx + off, f.vy + off,
                  f.vz + off, tile_end, f.tail0[is], f.ntail[is], part);
    EMSESG_LAUNCH(ctx, "fx_energy", k_fx_energy_sum, 1, 32, 0, part, DIAG_GRID, sum);
    double t[3];
    EMSESG_CUDA(ctx, cudaMemcpyAsync(t, sum, sizeof(t), cudaMemcpyDeviceToHost, ctx->stream));
    EMSESG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    // engk(d,is) = 0.5*rm(is)*t(d)/(slx*sly*slz), energy.F90:44-46
    for (int d = 0; d < 3; d++) engk[3 * is + d] = 0.5 * c.rm[is] * t[d] / vol;
  }
  return EMSESG_OK;
}

extern "C" int emsesg_fx_continuity(emsesg_ctx* ctx, double* res) {
  if (!ctx || !res) return EMSESG_ERR_ARG;
  if (!ctx->fx.loaded) return set_error(ctx, EMSESG_ERR_STATE, "FP32 form not loaded");
  FxState& f = ctx->fx;
  double r[2];
  EMSESG_CUDA(ctx, cudaMemcpyAsync(r, f.diag + 3 * DIAG_GRID + 3, sizeof(r), cudaMemcpyDeviceToHost, ctx->stream));
  EMSESG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  res[0] = f.cont_valid ? r[0] : std::nan("");
  res[1] = f.rho_prev ? r[1] : std::nan("");
  return EMSESG_OK;
}

extern "C" int emsesg_fx_background(emsesg_ctx* ctx, int replace) {
  if (!ctx) return EMSESG_ERR_ARG;
  if (!ctx->fx.loaded) return set_error(ctx, EMSESG_ERR_STATE, "FP32 form not loaded");
  const emsesg_config& c = ctx->cfg;
  FxState& f = ctx->fx;
  const FieldDesc fr = field_desc(c, EMSESG_FIELD_RHO);
  double* rhobk = ctx->field[EMSESG_FIELD_RHOBK];
  EMSESG_CUDA(ctx, cudaMemsetAsync(rhobk, 0, fr.size() * sizeof(double), ctx->stream));
  const Bodies bd = make_bodies(c);
  for (int is = 0; is < c.nspec; is++)
    for (int q = 0; q < bd.n; q++) {
      if (bd.kind[q] != 0) continue;  // the counts of box bodies only
      const int64_t nodes =
          (int64_t)(bd.hi[q][0] - bd.lo[q][0] + 1) * (bd.hi[q][1] - bd.lo[q][1] + 1) * (bd.hi[q][2] - bd.lo[q][2] + 1);
      EMSESG_LAUNCH(ctx, "fx_background", k_fx_background, nblk(nodes), 256, 0, f.surf + (int64_t)is * f.nsurf, bd,
                    q, c.q[is], rhobk, fr);
    }
  EMSESG_LAUNCH(ctx, "fx_background", k_add_background, nblk(fr.size()), 256, 0, ctx->field[EMSESG_FIELD_RHO],
                rhobk, fr, c.nx, c.ny, c.nz, replace ? 1 : 0);
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

namespace {

// Device copy of the FP32 state (particle arrays of every species region and
// the region layout) for the checkpoints of the adjoint.
struct FxSnap {
  float4* pos = nullptr;
  float* vx = nullptr;
  float* vy = nullptr;
  float* vz = nullptr;
  int64_t* ts = nullptr;
  int64_t* tp = nullptr;
  int64_t* counts = nullptr;  // count_d, slots_d
};

int snap_alloc(emsesg_ctx* ctx, FxSnap& sn, int64_t cap, int64_t nl) {
  EMSESG_CUDA(ctx, cudaMalloc(&sn.pos, cap * sizeof(float4)));
  EMSESG_CUDA(ctx, cudaMalloc(&sn.vx, cap * sizeof(float)));
  EMSESG_CUDA(ctx, cudaMalloc(&sn.vy, cap * sizeof(float)));
  EMSESG_CUDA(ctx, cudaMalloc(&sn.vz, cap * sizeof(float)));
  EMSESG_CUDA(ctx, cudaMalloc(&sn.ts, nl * sizeof(int64_t)));
  EMSESG_CUDA(ctx, cudaMalloc(&sn.tp, nl * sizeof(int64_t)));
  EMSESG_CUDA(ctx, cudaMalloc(&sn.counts, 2 * EMSESG_ISPEC * sizeof(int64_t)));
  return EMSESG_OK;
}

void snap_free(FxSnap& sn) {
  cudaFree(sn.pos); cudaFree(sn.vx); cudaFree(sn.vy); cudaFree(sn.vz);
  cudaFree(sn.ts); cudaFree(sn.tp); cudaFree(sn.counts);
  sn = FxSnap();
}

}  // namespace

// Buffers of emsesg_fx_adjoint, kept from call to call (allocating some
// thirty snapshots of the particle state costs more than a sweep) and
// released with the FP32 form.
struct emsesg::AdjWork {
  int64_t cap = 0, nl = 0, nn = 0;
  std::vector<FxSnap> ck, seg;     // checkpoints; the states of one segment
  std::vector<uint32_t*> inv;      // sort maps of one segment
  // the map of every sort of the forward pass, with the tile starts, tile
  // pads and counts after it (when they fit in memory): the recompute of a
  // segment applies them instead of sorting again
  std::vector<uint32_t*> maps;
  std::vector<int64_t*> meta;
  float *lam = nullptr, *lam2 = nullptr, *gd = nullptr;
  uint32_t* fwd = nullptr;  // a sort's old slot -> new slot
  double *gEd = nullptr, *gBd = nullptr;  // node-field gradients, FP64 sums
  float* jx = nullptr;             // probe Jx of each step
  int jx_steps = 0;
  double* lossd = nullptr;
  double* gvd = nullptr;
  int64_t gv_n = 0;
  void release() {
    for (auto& sn : ck) snap_free(sn);
    for (auto& sn : seg) snap_free(sn);
    for (auto* q : inv) cudaFree(q);
    for (auto* q : maps) cudaFree(q);
    for (auto* q : meta) cudaFree(q);
    cudaFree(lam); cudaFree(lam2); cudaFree(fwd); cudaFree(gd); cudaFree(gEd); cudaFree(gBd); cudaFree(jx);
    cudaFree(lossd); cudaFree(gvd);
    *this = AdjWork();
  }
};

void emsesg::adj_free(FxState& f) {
  if (f.adj) {
    f.adj->release();
    delete f.adj;
    f.adj = nullptr;
  }
}

namespace {

int adj_reserve(emsesg_ctx* ctx, AdjWork& w, int nseg, int ckpt, int jsteps, int64_t cap, int64_t nl, int64_t nn) {
  if (w.cap != cap || w.nl != nl || w.nn != nn) w.release();
  w.cap = cap; w.nl = nl; w.nn = nn;
  while ((int)w.ck.size() < nseg + 1) {
    w.ck.emplace_back();
    int rc = snap_alloc(ctx, w.ck.back(), cap, nl);
    if (rc) return rc;
  }
  while ((int)w.seg.size() < ckpt) {
    w.seg.emplace_back();
    int rc = snap_alloc(ctx, w.seg.back(), cap, nl);
    if (rc) return rc;
  }
  if ((int)w.inv.size() < ckpt) w.inv.resize((size_t)ckpt, nullptr);
  if (!w.lam) EMSESG_CUDA(ctx, cudaMalloc(&w.lam, 6 * cap * sizeof(float)));
  if (!w.lam2) EMSESG_CUDA(ctx, cudaMalloc(&w.lam2, 6 * cap * sizeof(float)));
  if (!w.fwd) EMSESG_CUDA(ctx, cudaMalloc(&w.fwd, cap * sizeof(uint32_t)));
  if (!w.gd) EMSESG_CUDA(ctx, cudaMalloc(&w.gd, 3 * nn * sizeof(float)));
  if (!w.gEd) EMSESG_CUDA(ctx, cudaMalloc(&w.gEd, 3 * nn * sizeof(double)));
  if (!w.gBd) EMSESG_CUDA(ctx, cudaMalloc(&w.gBd, 3 * nn * sizeof(double)));
  if (!w.lossd) EMSESG_CUDA(ctx, cudaMalloc(&w.lossd, sizeof(double)));
  if (w.jx_steps < jsteps) {
    cudaFree(w.jx);
    w.jx = nullptr;
    w.jx_steps = 0;
    EMSESG_CUDA(ctx, cudaMalloc(&w.jx, (size_t)jsteps * nn * sizeof(float)));
    w.jx_steps = jsteps;
  }
  return EMSESG_OK;
}

// Room for the maps of nsort sorts: taken when what is still to allocate
// is at most half of the free device memory (*keep), else the recompute
// sorts again.
int adj_reserve_maps(emsesg_ctx* ctx, AdjWork& w, int nsort, int64_t cap, int64_t nl, bool* keep) {
  *keep = false;
  const size_t mb = (size_t)cap * sizeof(uint32_t);
  const size_t tb = (size_t)(2 * nl + 2 * EMSESG_ISPEC) * sizeof(int64_t);
  const int have = (int)w.maps.size();
  if (have < nsort) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
      cudaGetLastError();
      return EMSESG_OK;
    }
    if ((size_t)(nsort - have) * (mb + tb) > fr / 2) return EMSESG_OK;
  }
  while ((int)w.maps.size() < nsort) {
    uint32_t* m = nullptr;
    int64_t* t = nullptr;
    EMSESG_CUDA(ctx, cudaMalloc(&m, mb));
    if (cudaMalloc(&t, tb) != cudaSuccess) {
      cudaFree(m);
      return check_cuda(ctx, cudaGetLastError(), "adjoint sort maps");
    }
    w.maps.push_back(m);
    w.meta.push_back(t);
  }
  *keep = true;
  return EMSESG_OK;
}

// Copies the live state into sn (save) or back; without `particles` only
// the tile starts and counts.
int snap_copy(emsesg_ctx* ctx, bool save, FxSnap& sn, int64_t cap, int64_t nl, bool particles = true) {
  FxState& f = ctx->fx;
  const cudaMemcpyKind k = cudaMemcpyDeviceToDevice;
  cudaStream_t st = ctx->stream;
#define EMSESG_SNAP(dst, src, bytes) EMSESG_CUDA(ctx, cudaMemcpyAsync(save ? (void*)(dst) : (void*)(src), \
                                                 save ? (const void*)(src) : (const void*)(dst), bytes, k, st))
  if (particles) {
    EMSESG_SNAP(sn.pos, f.pos, cap * sizeof(float4));
    EMSESG_SNAP(sn.vx, f.vx, cap * sizeof(float));
    EMSESG_SNAP(sn.vy, f.vy, cap * sizeof(float));
    EMSESG_SNAP(sn.vz, f.vz, cap * sizeof(float));
  }
  EMSESG_SNAP(sn.ts, f.tile_start, nl * sizeof(int64_t));
  EMSESG_SNAP(sn.tp, f.tile_pad, nl * sizeof(int64_t));
  EMSESG_SNAP(sn.counts, f.count_d, EMSESG_ISPEC * sizeof(int64_t));
  EMSESG_SNAP(sn.counts + EMSESG_ISPEC, f.slots_d, EMSESG_ISPEC * sizeof(int64_t));
#undef EMSESG_SNAP
  return EMSESG_OK;
}

// Puts the arrays o / o2 back into a / a2 (the live and the sort buffer),
// taking them from whichever holder (live, sort buffer, a segment state)
// has them: the recompute steps of the adjoint pass arrays around.
template <class T>
void reclaim(T*& a, T*& a2, T* o, T* o2, std::vector<FxSnap>& seg, T* FxSnap::*mem) {
  auto take = [&](T*& slot, T* want) {
    if (slot == want) return;
    if (a == want) { std::swap(slot, a); return; }
    if (a2 == want) { std::swap(slot, a2); return; }
    for (FxSnap& s : seg)
      if (s.*mem == want) { std::swap(slot, s.*mem); return; }
  };
  take(a, o);
  take(a2, o2);
}

// The particle arrays of the context as they were when the adjoint began;
// given back to their owners on every way out (the context frees them, and
// captured graphs hold their addresses).
struct ArrayOwners {
  FxState& f;
  std::vector<FxSnap>& seg;
  float4 *p0, *p1;
  float *x0, *x1, *y0, *y1, *z0, *z1;
  ArrayOwners(FxState& f_, std::vector<FxSnap>& s)
      : f(f_), seg(s), p0(f_.pos), p1(f_.pos2), x0(f_.vx), x1(f_.vx2), y0(f_.vy), y1(f_.vy2), z0(f_.vz),
        z1(f_.vz2) {}
  void give_back() {
    f.move_src = FxSrc{};
    reclaim(f.pos, f.pos2, p0, p1, seg, &FxSnap::pos);
    reclaim(f.vx, f.vx2, x0, x1, seg, &FxSnap::vx);
    reclaim(f.vy, f.vy2, y0, y1, seg, &FxSnap::vy);
    reclaim(f.vz, f.vz2, z0, z1, seg, &FxSnap::vz);
  }
  ~ArrayOwners() { give_back(); }
};

}  // namespace

extern "C" int emsesg_fx_adjoint(emsesg_ctx* ctx, int K, int ustep, int ckpt, int sort_every,
                                 const int32_t* probe_lo, const int32_t* probe_hi, double* loss, double* gE,
                                 double* gB, double* g0, double* gv) {
  if (!ctx || !probe_lo || !probe_hi || !loss) return EMSESG_ERR_ARG;
  FxState& f = ctx->fx;
  if (!f.loaded) return set_error(ctx, EMSESG_ERR_STATE, "FP32 form not loaded (emsesg_fx_load)");
  const emsesg_config& c = ctx->cfg;
  if (K < 1 || ckpt < 1 || ckpt > 64 || K % ckpt != 0 || ustep < 1 || sort_every < 1)
    return set_error(ctx, EMSESG_ERR_ARG, "adjoint: K >= 1 a multiple of ckpt (1..64), ustep, sort_every >= 1");
  for (int is = 0; is < c.nspec; is++) {
    for (int d = 0; d < 3; d++)
      if (c.npbnd[is][d] != 0) return set_error(ctx, EMSESG_ERR_UNSUPPORTED, "adjoint: periodic particles only");
    if (f.ntail[is]) return set_error(ctx, EMSESG_ERR_STATE, "adjoint: injected particles pending");
  }
  for (int d = 0; d < 3; d++)
    if (c.nfbnd[d] != 0) return set_error(ctx, EMSESG_ERR_UNSUPPORTED, "adjoint: periodic fields only");
  if (c.npc > 0 && c.line_mode != 1) return set_error(ctx, EMSESG_ERR_UNSUPPORTED, "adjoint: no bodies");
  int tmax = std::max(f.tile[0], std::max(f.tile[1], f.tile[2]));
  int64_t cap = 0;
  for (int is = 0; is < c.nspec; is++) cap += f.cap[is];
  const int64_t nl = (int64_t)c.nspec * (f.ntiles + 1);
  const int64_t nn = (int64_t)c.nx * c.ny * c.nz;
  const int nseg = K / ckpt;
  Geo g = make_geo(ctx);
  FieldDesc fj = field_desc(c, EMSESG_FIELD_AJ);
  const int3 lo = make_int3(probe_lo[0], probe_lo[1], probe_lo[2]);
  const int3 hi = make_int3(probe_hi[0], probe_hi[1], probe_hi[2]);
  // buffers (kept between calls): checkpoints, the states and sort maps of
  // one segment, lambda, g, node-field gradients, and the probe Jx of every
  // step, kept from the forward pass so that the recompute of a segment only
  // moves the particles (no rho / J)
  if (!f.adj) f.adj = new AdjWork();
  AdjWork& w = *f.adj;
  int rc = adj_reserve(ctx, w, nseg, ckpt, K, cap, nl, nn);
  if (rc) return rc;
  std::vector<FxSnap>& ck = w.ck;
  std::vector<FxSnap>& seg = w.seg;
  std::vector<uint32_t*>& inv = w.inv;
  float* lam = w.lam;
  float* lam2 = w.lam2;
  float* const jx = w.jx;
  float* const gd = w.gd;
  double* const gEd = w.gEd;
  double* const gBd = w.gBd;
  double* const lossd = w.lossd;
  bool keep_maps = false;
  rc = adj_reserve_maps(ctx, w, K / sort_every, cap, nl, &keep_maps);
  if (rc) return rc;
  ArrayOwners owners(f, seg);
  // the sort writes its map where f.lcs_inv points: a kept map for the
  // sorts of the forward pass, the context's own buffer again on every way out
  struct InvOwner {
    uint32_t*& p;
    uint32_t* const own;
    ~InvOwner() { p = own; }
  } inv_owner{f.lcs_inv, f.lcs_inv};
#define EMSESG_ADJ(call) do { rc = (call); if (rc) return rc; } while (0)
  EMSESG_ADJ(check_cuda(ctx, cudaMemsetAsync(lossd, 0, sizeof(double), ctx->stream), "adjoint loss"));
  // forward: K steps with a checkpoint every ckpt steps, the loss on the way
  for (int n = 0; n < K; n++) {
    if (n % ckpt == 0) EMSESG_ADJ(snap_copy(ctx, true, ck[(size_t)(n / ckpt)], cap, nl));
    const bool srt = (n + 1) % sort_every == 0;
    const int ks = (n + 1) / sort_every - 1;
    if (srt && keep_maps) {
      // slots past the new regions keep no map
      EMSESG_ADJ(check_cuda(ctx, cudaMemsetAsync(w.maps[(size_t)ks], 0xFF, cap * sizeof(uint32_t), ctx->stream),
                            "adjoint sort map"));
      f.lcs_inv = w.maps[(size_t)ks];
    }
    rc = emsesg_fx_step(ctx, ustep, srt ? 1 : 0);
    f.lcs_inv = inv_owner.own;
    if (rc) return rc;
    if (srt && keep_maps) {
      int64_t* t = w.meta[(size_t)ks];
      const cudaMemcpyKind dd = cudaMemcpyDeviceToDevice;
      EMSESG_CUDA(ctx, cudaMemcpyAsync(t, f.tile_start, nl * sizeof(int64_t), dd, ctx->stream));
      EMSESG_CUDA(ctx, cudaMemcpyAsync(t + nl, f.tile_pad, nl * sizeof(int64_t), dd, ctx->stream));
      EMSESG_CUDA(ctx, cudaMemcpyAsync(t + 2 * nl, f.count_d, EMSESG_ISPEC * sizeof(int64_t), dd, ctx->stream));
      EMSESG_CUDA(ctx, cudaMemcpyAsync(t + 2 * nl + EMSESG_ISPEC, f.slots_d, EMSESG_ISPEC * sizeof(int64_t), dd,
                                       ctx->stream));
    }
    EMSESG_LAUNCH(ctx, "adj_probe", k_adj_probe, nblk(nn), 256, 0, ctx->field[EMSESG_FIELD_AJ], fj, g, lo, hi,
                  lossd, jx + (int64_t)n * nn);
  }
  EMSESG_ADJ(snap_copy(ctx, true, ck[(size_t)nseg], cap, nl));  // the state after K steps, restored at the end
  // backward
  float* lx = lam;
  EMSESG_ADJ(check_cuda(ctx, cudaMemsetAsync(lam, 0, 6 * cap * sizeof(float), ctx->stream), "adjoint lambda"));
  EMSESG_ADJ(check_cuda(ctx, cudaMemsetAsync(gEd, 0, 3 * nn * sizeof(double), ctx->stream), "adjoint gE"));
  EMSESG_ADJ(check_cuda(ctx, cudaMemsetAsync(gBd, 0, 3 * nn * sizeof(double), ctx->stream), "adjoint gB"));
  AdjArgs a{};
  for (int is = 0; is < c.nspec; is++) {
    a.off[is] = f.base[is];
    a.qmp[is] = (float)(c.qm[is] * ustep * 0.5);
    a.q[is] = (float)c.q[is];
  }
  a.us = (float)ustep;
  a.rustep = (float)(1.0 / ustep);
  a.f0 = f.fnode;
  a.f1 = f.fnode2;
  a.g = gd;
  a.gE = gEd;
  a.gB = gBd;
  a.geo = g;
  a.ntiles = f.ntiles;
  const int asmem = fx_adjoint_smem(tmax);
  dim3 grid((unsigned)f.ntiles, (unsigned)c.nspec);
  for (int sgi = nseg - 1; sgi >= 0; sgi--) {
    EMSESG_ADJ(snap_copy(ctx, false, ck[(size_t)sgi], cap, nl));
    bool sorted[64] = {false};
    uint32_t* smap[64] = {nullptr};  // the map of the sort after step j
    for (int j = 0; j < ckpt; j++) {
      const int n = sgi * ckpt + j;
      // the state before step n is kept in seg[j]: its particle arrays take
      // the live ones (no copy), and the move-only step reads them and
      // writes the arrays seg[j] gave up
      FxSnap& sj = seg[(size_t)j];
      EMSESG_ADJ(snap_copy(ctx, true, sj, cap, nl, false));
      std::swap(f.pos, sj.pos);
      std::swap(f.vx, sj.vx);
      std::swap(f.vy, sj.vy);
      std::swap(f.vz, sj.vz);
      const bool srt = (n + 1) % sort_every == 0;
      const int ks = (n + 1) / sort_every - 1;
      const bool apply = srt && keep_maps;
      if (apply) {
        sorted[j] = true;
        smap[j] = w.maps[(size_t)ks];
      }
      // the state after the segment is not needed (only the map of a sort
      // after its last step, which is kept or made below)
      if (j == ckpt - 1 && (!srt || apply)) break;
      f.move_src = FxSrc{sj.pos, sj.vx, sj.vy, sj.vz};
      // slots past the new regions keep no map from an earlier sort
      if (srt && !apply)
        EMSESG_ADJ(check_cuda(ctx, cudaMemsetAsync(f.lcs_inv, 0xFF, cap * sizeof(uint32_t), ctx->stream), "inv"));
      EMSESG_ADJ(fx_step_impl(ctx, ustep, srt && !apply ? 1 : 0, false));
      f.move_src = FxSrc{};
      if (apply) {
        // the forward pass's sort again: gathered through its map, then its
        // tile starts, pads and counts
        for (int is = 0; is < c.nspec; is++) {
          const int64_t off = f.base[is];
          EMSESG_LAUNCH(ctx, "adj_apply", k_adj_apply, nblk(f.cap[is]), 256, 0, smap[j] + off, f.cap[is],
                        f.pos + off, f.vx + off, f.vy + off, f.vz + off, f.pos2 + off, f.vx2 + off, f.vy2 + off,
                        f.vz2 + off);
        }
        std::swap(f.pos, f.pos2);
        std::swap(f.vx, f.vx2);
        std::swap(f.vy, f.vy2);
        std::swap(f.vz, f.vz2);
        const int64_t* t = w.meta[(size_t)ks];
        const cudaMemcpyKind dd = cudaMemcpyDeviceToDevice;
        EMSESG_CUDA(ctx, cudaMemcpyAsync(f.tile_start, t, nl * sizeof(int64_t), dd, ctx->stream));
        EMSESG_CUDA(ctx, cudaMemcpyAsync(f.tile_pad, t + nl, nl * sizeof(int64_t), dd, ctx->stream));
        EMSESG_CUDA(ctx, cudaMemcpyAsync(f.count_d, t + 2 * nl, EMSESG_ISPEC * sizeof(int64_t), dd, ctx->stream));
        EMSESG_CUDA(ctx, cudaMemcpyAsync(f.slots_d, t + 2 * nl + EMSESG_ISPEC, EMSESG_ISPEC * sizeof(int64_t), dd,
                                         ctx->stream));
      } else if (srt && j < 64) {
        if (!inv[(size_t)j]) EMSESG_ADJ(check_cuda(ctx, cudaMalloc(&inv[(size_t)j], cap * sizeof(uint32_t)), "inv"));
        EMSESG_ADJ(check_cuda(ctx, cudaMemcpyAsync(inv[(size_t)j], f.lcs_inv, cap * sizeof(uint32_t),
                                                   cudaMemcpyDeviceToDevice, ctx->stream), "inv"));
        sorted[j] = true;
        smap[j] = inv[(size_t)j];
      }
    }
    for (int j = ckpt - 1; j >= 0; j--) {
      // lambda of S_{n+1}: in place, or across a re-sort after step n read
      // through the sort's forward map and written in the layout of S_n
      const bool across = j < 64 && sorted[j];
      float* lsrc = lx;
      if (across) {
        for (int is = 0; is < c.nspec; is++) {
          const int64_t off = f.base[is];
          EMSESG_LAUNCH(ctx, "adj_fwd", k_adj_fwd, nblk(f.cap[is]), 256, 0, smap[j] + off, f.cap[is],
                        w.fwd + off);
        }
        lx = lam2;
      }
      EMSESG_LAUNCH(ctx, "adj_g", k_adj_g, nblk(nn), 256, 0, jx + (int64_t)(sgi * ckpt + j) * nn, nn, gd);
      const FxSnap& sn = seg[(size_t)j];
      a.pos = sn.pos; a.vx = sn.vx; a.vy = sn.vy; a.vz = sn.vz;
      a.tile_start = sn.ts; a.tile_pad = sn.tp;
      a.lx = lx; a.ly = lx + cap; a.lz = lx + 2 * cap; a.lvx = lx + 3 * cap; a.lvy = lx + 4 * cap; a.lvz = lx + 5 * cap;
      a.slx = lsrc; a.sly = lsrc + cap; a.slz = lsrc + 2 * cap;
      a.slvx = lsrc + 3 * cap; a.slvy = lsrc + 4 * cap; a.slvz = lsrc + 5 * cap;
      a.fwd = across ? w.fwd : nullptr;
      if (fx_box_tile(tmax) == 4) {
        EMSESG_ADJ(check_cuda(ctx, cudaFuncSetAttribute(k_fx_adjoint<4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                        asmem), "adjoint smem"));
        EMSESG_LAUNCH(ctx, "fx_adjoint", k_fx_adjoint<4>, grid, ADJ_THREADS, asmem, a);
      } else {
        EMSESG_ADJ(check_cuda(ctx, cudaFuncSetAttribute(k_fx_adjoint<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                        asmem), "adjoint smem"));
        EMSESG_LAUNCH(ctx, "fx_adjoint", k_fx_adjoint<8>, grid, ADJ_THREADS, asmem, a);
      }
      if (across) {  // lambda_n went to lam2: it is the current lambda now
        std::swap(lam, lam2);
        lx = lam;
      }
    }
  }
  // outputs: lambda_v of the start state in canonical order, node gradients
  int64_t ntot = 0, rank0[EMSESG_ISPEC];
  int64_t cnt0[2 * EMSESG_ISPEC];
  EMSESG_ADJ(check_cuda(ctx, cudaMemcpyAsync(cnt0, ck[0].counts, sizeof(cnt0), cudaMemcpyDeviceToHost, ctx->stream),
                        "counts"));
  EMSESG_ADJ(check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "sync"));
  for (int is = 0; is < c.nspec; is++) { rank0[is] = ntot; ntot += cnt0[is]; }
  if (gv) {
    if (w.gv_n < ntot) {
      cudaFree(w.gvd);
      w.gvd = nullptr;
      w.gv_n = 0;
      EMSESG_ADJ(check_cuda(ctx, cudaMalloc(&w.gvd, std::max<int64_t>(ntot, 1) * 3 * sizeof(double)), "gv"));
      w.gv_n = ntot;
    }
    double* const gvd = w.gvd;
    for (int is = 0; is < c.nspec; is++) {
      const int64_t off = f.base[is];
      EMSESG_LAUNCH(ctx, "adj_canonical", k_adj_canonical, (unsigned)f.ntiles, PUSH_THREADS, 0, lx + 3 * cap + off,
                    lx + 4 * cap + off, lx + 5 * cap + off, ck[0].ts + (int64_t)is * (f.ntiles + 1),
                    ck[0].tp + (int64_t)is * (f.ntiles + 1), rank0[is], gvd);
    }
    EMSESG_ADJ(check_cuda(ctx, cudaMemcpyAsync(gv, gvd, ntot * 3 * sizeof(double), cudaMemcpyDeviceToHost,
                                               ctx->stream), "gv"));
  }
  std::vector<double> hE((size_t)(3 * nn)), hB((size_t)(3 * nn));
  EMSESG_ADJ(check_cuda(ctx, cudaMemcpyAsync(hE.data(), gEd, 3 * nn * sizeof(double), cudaMemcpyDeviceToHost,
                                             ctx->stream), "gE"));
  EMSESG_ADJ(check_cuda(ctx, cudaMemcpyAsync(hB.data(), gBd, 3 * nn * sizeof(double), cudaMemcpyDeviceToHost,
                                             ctx->stream), "gB"));
  EMSESG_ADJ(check_cuda(ctx, cudaMemcpyAsync(loss, lossd, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream),
                        "loss"));
  owners.give_back();
  EMSESG_ADJ(snap_copy(ctx, false, ck[(size_t)nseg], cap, nl));
  EMSESG_ADJ(check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "sync"));
  double s0[6] = {0, 0, 0, 0, 0, 0};
  for (int64_t u = 0; u < nn; u++)
    for (int k = 0; k < 3; k++) {
      s0[k] += hE[(size_t)(3 * u + k)];
      s0[3 + k] += hB[(size_t)(3 * u + k)];
      if (gE) gE[3 * u + k] = hE[(size_t)(3 * u + k)];
      if (gB) gB[3 * u + k] = hB[(size_t)(3 * u + k)];
    }
  if (g0)
    for (int k = 0; k < 6; k++) g0[k] = s0[k];
  // lambda buffers swap in the sweep: keep them with the workspace
  w.lam = lam;
  w.lam2 = lam2;
#undef EMSESG_ADJ
  return emsesg_synchronize(ctx);
}

namespace {

// Captures `block` steps of ctx (do_sort on every sort_every-th) into a new
// graph.  Capturing runs no kernel; the host state that the steps touch
// (buffer swaps of the sorts, the step counter of the random hash) is
// checked, or put back, so that it matches the state after a replay.
int capture_steps(emsesg_ctx* ctx, int ustep, int block, int sort_every, cudaGraph_t* out) {
  FxState& f = ctx->fx;
  *out = nullptr;
  const bool timing = ctx->timer.on;
  float4* pos0 = f.pos;
  const int64_t* ts0 = f.tile_start;
  const uint64_t rs0 = ctx->rng_stream;
  ctx->timer.on = false;
  EMSESG_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  f.capture = true;
  int rc = EMSESG_OK;
  for (int s = 0; s < block && !rc; s++) rc = emsesg_fx_step(ctx, ustep, (s + 1) % sort_every == 0);
  f.capture = false;
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
  ctx->timer.on = timing;
  ctx->rng_stream = rs0;
  if (rc) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (e != cudaSuccess) return check_cuda(ctx, e, "cudaStreamEndCapture");
  if (f.pos != pos0 || f.tile_start != ts0) {
    cudaGraphDestroy(graph);
    return set_error(ctx, EMSESG_ERR_STATE, "captured block does not return to its buffers");
  }
  *out = graph;
  return EMSESG_OK;
}

bool graph_ready(const emsesg_ctx* ctx) {
  const FxState& f = ctx->fx;
  bool tail = false;
  for (int is = 0; is < ctx->cfg.nspec; is++) tail = tail || f.ntail[is] > 0 || f.pending[is] > 0;
  return f.tiled && !tail && !f.inj_j_pending;
}

}  // namespace

// nsteps steps of the FP32 form with a re-sort every sort_every steps.  With
// use_graph the block of 2*sort_every steps (two sorts, so that the buffer
// swaps of the sorts cancel) is captured once into a CUDA graph and replayed;
// steps that do not fill a block run one by one.  Asynchronous.
extern "C" int emsesg_fx_run(emsesg_ctx* ctx, int ustep, int nsteps, int sort_every, int use_graph) {
  if (!ctx || nsteps < 0 || sort_every < 1) return EMSESG_ERR_ARG;
  FxState& f = ctx->fx;
  if (!f.loaded) return set_error(ctx, EMSESG_ERR_STATE, "FP32 form not loaded (emsesg_fx_load)");
  // a pending asynchronous eb upload is taken now, outside any capture
  int rc = apply_pending_eb(ctx);
  if (rc) return rc;
  const int block = 2 * sort_every;
  if (!use_graph || !graph_ready(ctx) || nsteps < block) {
    for (int s = 0; s < nsteps; s++)
      if ((rc = emsesg_fx_step(ctx, ustep, (s + 1) % sort_every == 0))) return rc;
    return EMSESG_OK;
  }
  if (f.gexec && (f.g_ustep != ustep || f.g_sort != sort_every || f.g_pos != f.pos || f.g_ts != f.tile_start ||
                  f.g_eb != ctx->field[EMSESG_FIELD_EB] || memcmp(&f.g_cfg, &ctx->cfg, sizeof(emsesg_config)) != 0)) {
    cudaGraphExecDestroy(f.gexec);
    f.gexec = nullptr;
  }
  if (!f.gexec) {
    cudaGraph_t graph;
    if ((rc = capture_steps(ctx, ustep, block, sort_every, &graph))) return rc;
    cudaError_t e = cudaGraphInstantiate(&f.gexec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      f.gexec = nullptr;
      return check_cuda(ctx, e, "cudaGraphInstantiate");
    }
    f.g_ustep = ustep;
    f.g_sort = sort_every;
    f.g_pos = f.pos;
    f.g_ts = f.tile_start;
    f.g_eb = ctx->field[EMSESG_FIELD_EB];
    f.g_cfg = ctx->cfg;
  }
  const int nblock = nsteps / block;
  for (int b = 0; b < nblock; b++) EMSESG_CUDA(ctx, cudaGraphLaunch(f.gexec, ctx->stream));
  if (ctx->ev_fields) EMSESG_CUDA(ctx, cudaEventRecord(ctx->ev_fields, ctx->stream));
  ctx->rng_stream += (uint64_t)nblock * block;
  for (int s = 0; s < nsteps - nblock * block; s++)
    if ((rc = emsesg_fx_step(ctx, ustep, (s + 1) % sort_every == 0))) return rc;
  return EMSESG_OK;
}

// ---- ensembles: one graph holding a block of steps of many runs ----------
// Each run (context) is captured on its own stream into a child graph; the
// children sit side by side in one parent graph with no edges between them,
// so one cudaGraphLaunch starts every run and the GPU runs their kernels
// concurrently, small runs filling the SMs that one run leaves idle.
struct emsesg_batch {
  std::vector<emsesg_ctx*> ctxs;
  std::vector<cudaEvent_t> ev;      // one per context: its stream's last work
  std::vector<float4*> pos;         // buffers each run was captured with
  std::vector<const int64_t*> ts;
  std::vector<const double*> eb;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  cudaGraphExec_t exec = nullptr;
  int block = 0;
  int64_t kernels = 0;              // kernel nodes in one replay
};

extern "C" int emsesg_batch_destroy(emsesg_batch* b) {
  if (!b) return EMSESG_OK;
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  for (cudaEvent_t e : b->ev) cudaEventDestroy(e);
  if (b->done) cudaEventDestroy(b->done);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return EMSESG_OK;
}

extern "C" int emsesg_batch_create(emsesg_ctx* const* ctxs, int n, int ustep, int block, const int* sort_every,
                                   emsesg_batch** out) {
  if (!ctxs || n < 1 || !sort_every || !out || block < 2) return EMSESG_ERR_ARG;
  *out = nullptr;
  emsesg_ctx* c0 = ctxs[0];
  if (!c0) return EMSESG_ERR_ARG;
  for (int r = 0; r < n; r++) {
    emsesg_ctx* c = ctxs[r];
    if (!c) return EMSESG_ERR_ARG;
    for (int q = 0; q < r; q++)
      if (ctxs[q] == c) return set_error(c, EMSESG_ERR_ARG, "a context appears twice in the batch");
    if (c->device != c0->device) return set_error(c, EMSESG_ERR_ARG, "batch contexts must share one device");
    if (sort_every[r] < 1 || block % (2 * sort_every[r]) != 0)
      return set_error(c, EMSESG_ERR_ARG, "block %d is not a multiple of 2*sort_every (%d)", block, sort_every[r]);
    if (!c->fx.loaded) return set_error(c, EMSESG_ERR_STATE, "FP32 form not loaded (emsesg_fx_load)");
    if (!graph_ready(c)) return set_error(c, EMSESG_ERR_STATE, "run is not tile-sorted or has injected particles");
    // a pending asynchronous eb upload is taken before the capture
    int rc0 = apply_pending_eb(c);
    if (rc0) return rc0;
  }
  emsesg_batch* b = new emsesg_batch();
  b->ctxs.assign(ctxs, ctxs + n);
  b->block = block;
  int rc = EMSESG_OK;
  cudaGraph_t parent = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaGraphCreate(&parent, 0);
  for (int r = 0; r < n && e == cudaSuccess; r++) {
    cudaEvent_t ev;
    e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e == cudaSuccess) b->ev.push_back(ev);
  }
  if (e != cudaSuccess) rc = check_cuda(c0, e, "batch resources");
  for (int r = 0; r < n && !rc; r++) {
    cudaGraph_t child = nullptr;
    if ((rc = capture_steps(ctxs[r], ustep, block, sort_every[r], &child))) break;
    size_t nn = 0;
    e = cudaGraphGetNodes(child, nullptr, &nn);
    if (e == cudaSuccess && nn) {
      std::vector<cudaGraphNode_t> nodes(nn);
      e = cudaGraphGetNodes(child, nodes.data(), &nn);
      for (size_t q = 0; q < nn && e == cudaSuccess; q++) {
        cudaGraphNodeType t;
        e = cudaGraphNodeGetType(nodes[q], &t);
        if (t == cudaGraphNodeTypeKernel) b->kernels++;
      }
    }
    cudaGraphNode_t node;
    if (e == cudaSuccess) e = cudaGraphAddChildGraphNode(&node, parent, nullptr, 0, child);
    cudaGraphDestroy(child);
    if (e != cudaSuccess) rc = check_cuda(ctxs[r], e, "cudaGraphAddChildGraphNode");
    b->pos.push_back(ctxs[r]->fx.pos);
    b->ts.push_back(ctxs[r]->fx.tile_start);
    b->eb.push_back(ctxs[r]->field[EMSESG_FIELD_EB]);
  }
  if (!rc) {
    e = cudaGraphInstantiate(&b->exec, parent, 0);
    if (e != cudaSuccess) {
      b->exec = nullptr;
      rc = check_cuda(c0, e, "cudaGraphInstantiate");
    }
  }
  if (parent) cudaGraphDestroy(parent);
  if (rc) {
    emsesg_batch_destroy(b);
    return rc;
  }
  *out = b;
  return EMSESG_OK;
}

extern "C" int emsesg_batch_launch(emsesg_batch* b, int nrep) {
  if (!b || nrep < 0) return EMSESG_ERR_ARG;
  emsesg_ctx* c0 = b->ctxs[0];
  const int n = (int)b->ctxs.size();
  for (int r = 0; r < n; r++) {
    emsesg_ctx* c = b->ctxs[r];
    if (c->fx.pos != b->pos[r] || c->fx.tile_start != b->ts[r] || graph_ready(c) == false)
      return set_error(c, EMSESG_ERR_STATE, "run changed since the batch was captured");
    // the graph reads the eb buffer it was captured with; an asynchronous
    // upload goes to the other one
    if (c->eb_next_pending || c->field[EMSESG_FIELD_EB] != b->eb[r])
      return set_error(c, EMSESG_ERR_STATE, "eb uploaded asynchronously since the batch was captured");
  }
  // the graph starts after each run's earlier work ...
  for (int r = 0; r < n; r++) {
    EMSESG_CUDA(c0, cudaEventRecord(b->ev[r], b->ctxs[r]->stream));
    EMSESG_CUDA(c0, cudaStreamWaitEvent(b->stream, b->ev[r], 0));
  }
  for (int k = 0; k < nrep; k++) EMSESG_CUDA(c0, cudaGraphLaunch(b->exec, b->stream));
  // ... and each run's later work starts after the graph
  EMSESG_CUDA(c0, cudaEventRecord(b->done, b->stream));
  for (int r = 0; r < n; r++) {
    EMSESG_CUDA(c0, cudaStreamWaitEvent(b->ctxs[r]->stream, b->done, 0));
    b->ctxs[r]->rng_stream += (uint64_t)nrep * b->block;
    // the graph's reads of eb are over once the run's stream gets here
    if (b->ctxs[r]->ev_fields) EMSESG_CUDA(c0, cudaEventRecord(b->ctxs[r]->ev_fields, b->ctxs[r]->stream));
  }
  return EMSESG_OK;
}

extern "C" void* emsesg_batch_stream(emsesg_batch* b) { return b ? (void*)b->stream : nullptr; }

extern "C" int emsesg_batch_kernels(const emsesg_batch* b, int64_t* n) {
  if (!b || !n) return EMSESG_ERR_ARG;
  *n = b->kernels;
  return EMSESG_OK;
}
