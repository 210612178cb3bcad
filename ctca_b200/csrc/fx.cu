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
// charge of charge.F90:59-80 at the new position.  Deposits are summed over
// the lanes of a warp that share a cell (a fixed 32-lane reduction tree),
// converted to int64 fixed point at 2^40 and added into a shared-memory
// accumulator covering the tile plus a 2-cell guard; the CTA then adds its
// accumulator into the global int64 arrays.  Integer adds commute, so the
// global sums do not depend on the order in which CTAs and atomics run.
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "slab.cuh"

namespace emsesg {

namespace {

constexpr uint32_t DEAD = 0xFFFFFFFFu;
constexpr int FX_THREADS = 256;
constexpr int GUARD = 2;
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
struct FxPushArgs {
  float4* pos;
  float* vx;
  float* vy;
  float* vz;
  const int64_t* tile_start;  // this species, ntiles+1 entries
  const float4* __restrict__ f0;
  const float4* __restrict__ f1;
  unsigned long long* acc_rho;  // rho layout (1, -1:n+1)
  unsigned long long* acc_j;    // aj layout (3, -4:n+4)
  FieldDesc fr, fj;
  Geo g;
  int npbnd[3];
  float qmp, gustep, rustep, qfix;  // qfix = q * 2^40
  int* nesc;
  int* status;
  long long* diag;
};

// Per-axis move and outer boundary of psolve1.F90:366-606 on (cell, offset)
// pairs.  In: cell ib, offset ob, displacement d.  Out: the "after" point
// xlocala = (ac, af), its cell ia, the relay point xr = (rc, rf), the stored
// new position (nc, nf), and flags.
struct Axis {
  int ac, ia, rc, nc;
  float af, rf, nf;
  bool dead, flip, crossed;
};

__device__ __forceinline__ Axis axis_move(int ib, float ob, float d, int n, int npbnd) {
  Axis o;
  float s = ob + d;
  float fl = floorf(s);
  int ac = ib + (int)fl;
  float af = s - fl;
  if (af >= 1.0f) { af = 0.0f; ac += 1; }
  o.dead = false;
  o.flip = false;
  o.crossed = false;
  if (ac < 0) {  // p%x < 0
    o.crossed = true;
    if (npbnd == 0) {
      o.ac = ac; o.af = af; o.ia = -1; o.rc = 0; o.rf = 0.f;
      o.nc = ac + n; o.nf = af;
    } else if (npbnd == 1) {
      int rc_ = af > 0.f ? -ac - 1 : -ac;
      float rf_ = af > 0.f ? 1.0f - af : 0.0f;
      if (rf_ >= 1.0f) { rf_ = 0.f; rc_ += 1; }
      o.ac = rc_; o.af = rf_; o.ia = 0; o.rc = 0; o.rf = 0.f;
      o.nc = rc_; o.nf = rf_; o.flip = true;
    } else {
      o.ac = -1; o.af = 0.f; o.ia = -1; o.rc = 0; o.rf = 0.f;
      o.nc = 0; o.nf = 0.f; o.dead = true;
    }
  } else if (ac >= n) {  // p%x >= slx
    o.crossed = true;
    if (npbnd == 0) {
      o.ac = ac; o.af = af; o.ia = n; o.rc = n; o.rf = 0.f;
      o.nc = ac - n; o.nf = af;
    } else if (npbnd == 1) {
      int rc_ = af > 0.f ? 2 * n - ac - 1 : 2 * n - ac;
      float rf_ = af > 0.f ? 1.0f - af : 0.0f;
      if (rf_ >= 1.0f) { rf_ = 0.f; rc_ += 1; }
      o.ac = rc_; o.af = rf_; o.ia = n - 1; o.rc = n; o.rf = 0.f;
      o.nc = rc_; o.nf = rf_; o.flip = true;
    } else {
      o.ac = n + 1; o.af = 0.f; o.ia = n; o.rc = n; o.rf = 0.f;
      o.nc = 0; o.nf = 0.f; o.dead = true;
    }
  } else {
    o.ac = ac; o.af = af; o.ia = ac;
    if (ac == ib) { o.rc = ib; o.rf = (ob + af) * 0.5f; }
    else { o.rc = max(ib, ac); o.rf = 0.f; }
    o.nc = ac; o.nf = af;
  }
  return o;
}

// Slot layout of the 20 merged deposits of one cell: 0-3 JX at (0,dj,dk),
// 4-7 JY at (di,0,dk), 8-11 JZ at (di,dj,0) with (d1,d2) = (s&1, (s>>1)&1),
// 12-19 rho at the CIC corners in charge.F90 order v1..v8.
__device__ __forceinline__ void slot_offset(int s, int& comp, int& di, int& dj, int& dk) {
  if (s < 12) {
    int a = s & 1, b = (s >> 1) & 1;
    comp = 1 + (s >> 2);
    if (s < 4) { di = 0; dj = a; dk = b; }
    else if (s < 8) { di = a; dj = 0; dk = b; }
    else { di = a; dj = b; dk = 0; }
  } else {
    // v1..v8 corners: (0,0,1) (1,0,1) (1,1,1) (0,1,1) (0,0,0) (1,0,0) (1,1,0) (0,1,0)
    int r = s - 12, q = r & 3;
    comp = 0;
    di = (q == 1 || q == 2) ? 1 : 0;
    dj = q >= 2 ? 1 : 0;
    dk = r < 4 ? 1 : 0;
  }
}

struct Box {
  int o[3];   // global index of box entry 0
  int B;      // entries per axis
};

__device__ __forceinline__ bool in_box(const Box& bx, int i, int j, int k) {
  return i >= bx.o[0] && j >= bx.o[1] && k >= bx.o[2] && i + 1 < bx.o[0] + bx.B && j + 1 < bx.o[1] + bx.B &&
         k + 1 < bx.o[2] + bx.B;
}

__device__ __forceinline__ void deposit_one(const FxPushArgs& a, const Box& bx, unsigned long long* box, int comp,
                                            int i, int j, int k, long long v, bool inbox) {
  if (v == 0) return;
  if (inbox) {
    int li = i - bx.o[0], lj = j - bx.o[1], lk = k - bx.o[2];
    atomicAdd(&box[((comp * bx.B + lk) * bx.B + lj) * bx.B + li], (unsigned long long)v);
  } else if (comp == 0) {
    if (i < -1 || j < -1 || k < -1 || i > a.g.nx + 1 || j > a.g.ny + 1 || k > a.g.nz + 1) {
      report_bad(a.status, a.diag, SITE_FX_DEPOSIT, -1, i + 100000LL * j + 10000000000LL * k);
      return;
    }
    atomicAdd(&a.acc_rho[a.fr.at(0, i, j, k)], (unsigned long long)v);
  } else {
    if (i < -4 || j < -4 || k < -4 || i > a.g.nx + 4 || j > a.g.ny + 4 || k > a.g.nz + 4) {
      report_bad(a.status, a.diag, SITE_FX_DEPOSIT, -2, i + 100000LL * j + 10000000000LL * k);
      return;
    }
    atomicAdd(&a.acc_j[a.fj.at(comp - 1, i, j, k)], (unsigned long long)v);
  }
}

__device__ __forceinline__ long long to_fix(float v, float scale) { return __float2ll_rn(v * scale); }

// 32 lanes x 32 values -> lane L holds the sum over lanes of value L.
// Fixed butterfly tree: the result does not depend on scheduling.
__device__ __forceinline__ float transpose_reduce(float (&v)[32], int lane) {
#pragma unroll
  for (int h = 16; h >= 1; h >>= 1) {
    bool upper = (lane & h) != 0;
#pragma unroll
    for (int i = 0; i < h; i++) {
      float send = upper ? v[i] : v[i + h];
      float keep = upper ? v[i + h] : v[i];
      float recv = __shfl_xor_sync(0xffffffffu, send, h);
      v[i] = keep + recv;
    }
  }
  return v[0];
}

__global__ void __launch_bounds__(FX_THREADS) k_fx_push(FxPushArgs a) {
  extern __shared__ unsigned long long box[];
  const Geo& g = a.g;
  int t = blockIdx.x;
  int tx = t % g.nt[0], ty = (t / g.nt[0]) % g.nt[1], tz = t / (g.nt[0] * g.nt[1]);
  Box bx;
  bx.o[0] = tx * g.t[0] - GUARD;
  bx.o[1] = ty * g.t[1] - GUARD;
  bx.o[2] = tz * g.t[2] - GUARD;
  bx.B = max(g.t[0], max(g.t[1], g.t[2])) + 2 * GUARD + 1;
  const int nbox = 4 * bx.B * bx.B * bx.B;
  for (int e = threadIdx.x; e < nbox; e += blockDim.x) box[e] = 0ull;
  __syncthreads();

  const int lane = threadIdx.x & 31;
  int64_t p0 = a.tile_start[t], p1 = a.tile_start[t + 1];
  for (int64_t base = p0; base < p1; base += blockDim.x) {
    int64_t m = base + threadIdx.x;
    bool inrange = m < p1;
    float4 ps = inrange ? a.pos[m] : make_float4(0.f, 0.f, 0.f, __int_as_float((int)DEAD));
    uint32_t cell = (uint32_t)__float_as_int(ps.w);
    bool live = inrange && cell != DEAD;
    float vx = 0.f, vy = 0.f, vz = 0.f;
    if (live) { vx = a.vx[m]; vy = a.vy[m]; vz = a.vz[m]; }
    int ib = 0, jb = 0, kb = 0;
    if (live) {
      unpack(g, cell, ib, jb, kb);
      if (ib >= g.nx || jb >= g.ny || kb >= g.nz) {
        report_bad(a.status, a.diag, SITE_FX_PUSH, m, (long long)cell);
        live = false;
      }
    }
    float J1[12], J2[12], R[8];
    Axis ax{}, ay{}, az{};
    bool dead = false;
    if (live) {
      // trilinear weights (psolve1.F90:186-199)
      float x1 = ps.x, y1 = ps.y, z1 = ps.z;
      float xy1 = x1 * y1, xz1 = x1 * z1, yz1 = y1 * z1, z2 = 1.0f - z1;
      float xz2 = x1 * z2, yz2 = y1 * z2;
      float v3 = xy1 * z1, v2 = xz1 - v3, v4 = yz1 - v3, v1 = z1 - xz1 - v4;
      float v7 = xy1 * z2, v6 = xz2 - v7, v8 = yz2 - v7, v5 = z2 - xz2 - v8;
      int64_t sy = g.nx + 1, sz = (int64_t)(g.nx + 1) * (g.ny + 1);
      int64_t n5 = ib + sy * jb + sz * kb, n1 = n5 + sz;
      float4 a1 = __ldg(&a.f0[n1]), a2 = __ldg(&a.f0[n1 + 1]), a3 = __ldg(&a.f0[n1 + 1 + sy]), a4 = __ldg(&a.f0[n1 + sy]);
      float4 a5 = __ldg(&a.f0[n5]), a6 = __ldg(&a.f0[n5 + 1]), a7 = __ldg(&a.f0[n5 + 1 + sy]), a8 = __ldg(&a.f0[n5 + sy]);
      float4 b1 = __ldg(&a.f1[n1]), b2 = __ldg(&a.f1[n1 + 1]), b3 = __ldg(&a.f1[n1 + 1 + sy]), b4 = __ldg(&a.f1[n1 + sy]);
      float4 b5 = __ldg(&a.f1[n5]), b6 = __ldg(&a.f1[n5 + 1]), b7 = __ldg(&a.f1[n5 + 1 + sy]), b8 = __ldg(&a.f1[n5 + sy]);
      float eex = a1.x * v1 + a2.x * v2 + a3.x * v3 + a4.x * v4 + a5.x * v5 + a6.x * v6 + a7.x * v7 + a8.x * v8;
      float eey = a1.y * v1 + a2.y * v2 + a3.y * v3 + a4.y * v4 + a5.y * v5 + a6.y * v6 + a7.y * v7 + a8.y * v8;
      float eez = a1.z * v1 + a2.z * v2 + a3.z * v3 + a4.z * v4 + a5.z * v5 + a6.z * v6 + a7.z * v7 + a8.z * v8;
      float bbx = a1.w * v1 + a2.w * v2 + a3.w * v3 + a4.w * v4 + a5.w * v5 + a6.w * v6 + a7.w * v7 + a8.w * v8;
      float bby = b1.x * v1 + b2.x * v2 + b3.x * v3 + b4.x * v4 + b5.x * v5 + b6.x * v6 + b7.x * v7 + b8.x * v8;
      float bbz = b1.y * v1 + b2.y * v2 + b3.y * v3 + b4.y * v4 + b5.y * v5 + b6.y * v6 + b7.y * v7 + b8.y * v8;
      // Buneman-Boris (psolve1.F90:247-272)
      eex *= a.qmp; eey *= a.qmp; eez *= a.qmp;
      bbx *= a.qmp; bby *= a.qmp; bbz *= a.qmp;
      float boris = 2.0f / (1.0f + bbx * bbx + bby * bby + bbz * bbz);
      vx += eex; vy += eey; vz += eez;
      float vxt = vx + vy * bbz - vz * bby;
      float vyt = vy + vz * bbx - vx * bbz;
      float vzt = vz + vx * bby - vy * bbx;
      vx += boris * (vyt * bbz - vzt * bby);
      vy += boris * (vzt * bbx - vxt * bbz);
      vz += boris * (vxt * bby - vyt * bbx);
      vx += eex; vy += eey; vz += eez;
      // move + outer boundary per axis
      ax = axis_move(ib, ps.x, vx * a.gustep, g.nx, a.npbnd[0]);
      ay = axis_move(jb, ps.y, vy * a.gustep, g.ny, a.npbnd[1]);
      az = axis_move(kb, ps.z, vz * a.gustep, g.nz, a.npbnd[2]);
      if (ax.flip) vx = -vx;
      if (ay.flip) vy = -vy;
      if (az.flip) vz = -vz;
      dead = ax.dead || ay.dead || az.dead;
      // zigzag (psolve1.F90:717-757), differences taken on integers first
      float xd1 = ((float)(ax.rc - ib) + ax.rf + ps.x) * 0.5f;
      float yd1 = ((float)(ay.rc - jb) + ay.rf + ps.y) * 0.5f;
      float zd1 = ((float)(az.rc - kb) + az.rf + ps.z) * 0.5f;
      float vvx1 = ((float)(ax.rc - ib) + (ax.rf - ps.x)) * a.rustep;
      float vvy1 = ((float)(ay.rc - jb) + (ay.rf - ps.y)) * a.rustep;
      float vvz1 = ((float)(az.rc - kb) + (az.rf - ps.z)) * a.rustep;
      float xd2 = ((float)(ax.ac - ax.ia) + ax.af + (float)(ax.rc - ax.ia) + ax.rf) * 0.5f;
      float yd2 = ((float)(ay.ac - ay.ia) + ay.af + (float)(ay.rc - ay.ia) + ay.rf) * 0.5f;
      float zd2 = ((float)(az.ac - az.ia) + az.af + (float)(az.rc - az.ia) + az.rf) * 0.5f;
      float vvx2 = ((float)(ax.ac - ax.rc) + (ax.af - ax.rf)) * a.rustep;
      float vvy2 = ((float)(ay.ac - ay.rc) + (ay.af - ay.rf)) * a.rustep;
      float vvz2 = ((float)(az.ac - az.rc) + (az.af - az.rf)) * a.rustep;
      float w;
      w = yd1 * zd1; J1[3] = vvx1 * w; J1[1] = vvx1 * (yd1 - w); J1[2] = vvx1 * (zd1 - w); J1[0] = vvx1 * (1.0f - yd1 - (zd1 - w));
      w = xd1 * zd1; J1[7] = vvy1 * w; J1[5] = vvy1 * (xd1 - w); J1[6] = vvy1 * (zd1 - w); J1[4] = vvy1 * (1.0f - xd1 - (zd1 - w));
      w = xd1 * yd1; J1[11] = vvz1 * w; J1[9] = vvz1 * (xd1 - w); J1[10] = vvz1 * (yd1 - w); J1[8] = vvz1 * (1.0f - xd1 - (yd1 - w));
      w = yd2 * zd2; J2[3] = vvx2 * w; J2[1] = vvx2 * (yd2 - w); J2[2] = vvx2 * (zd2 - w); J2[0] = vvx2 * (1.0f - yd2 - (zd2 - w));
      w = xd2 * zd2; J2[7] = vvy2 * w; J2[5] = vvy2 * (xd2 - w); J2[6] = vvy2 * (zd2 - w); J2[4] = vvy2 * (1.0f - xd2 - (zd2 - w));
      w = xd2 * yd2; J2[11] = vvz2 * w; J2[9] = vvz2 * (xd2 - w); J2[10] = vvz2 * (yd2 - w); J2[8] = vvz2 * (1.0f - xd2 - (yd2 - w));
      // CIC rho at the stored position (charge.F90:173-209)
      if (!dead) {
        float X = ax.nf, Y = ay.nf, Z = az.nf;
        float XY = X * Y, XZ = X * Z, YZ = Y * Z, Z2 = 1.0f - Z, XZ2 = X * Z2, YZ2 = Y * Z2;
        R[2] = XY * Z; R[1] = XZ - R[2]; R[3] = YZ - R[2]; R[0] = Z - XZ - R[3];
        R[6] = XY * Z2; R[5] = XZ2 - R[6]; R[7] = YZ2 - R[6]; R[4] = Z2 - XZ2 - R[7];
      } else {
#pragma unroll
        for (int r = 0; r < 8; r++) R[r] = 0.f;
        atomicAdd(a.nesc, 1);
      }
      // store
      uint32_t nc = dead ? DEAD : pack(g, ax.nc, ay.nc, az.nc);
      a.pos[m] = make_float4(ax.nf, ay.nf, az.nf, __int_as_float((int)nc));
      a.vx[m] = vx; a.vy[m] = vy; a.vz[m] = vz;
    } else {
#pragma unroll
      for (int r = 0; r < 12; r++) { J1[r] = 0.f; J2[r] = 0.f; }
#pragma unroll
      for (int r = 0; r < 8; r++) R[r] = 0.f;
    }

    // ---- deposit
    // "simple" lanes: no cell change, no boundary event: all 20 merged
    // values sit at one base cell.
    bool simple = live && !ax.crossed && !ay.crossed && !az.crossed && ax.ia == ib && ay.ia == jb && az.ia == kb;
    uint32_t key = simple ? cell : DEAD;
    unsigned sb = __ballot_sync(0xffffffffu, simple);
    bool done = !simple;  // lanes whose merged deposit is still pending
    for (int grp = 0; grp < 2 && sb; grp++) {
      int leader = grp == 0 ? __ffs(sb) - 1 : 31 - __clz(sb);
      uint32_t gkey = __shfl_sync(0xffffffffu, key, leader);
      bool mem = simple && !done && key == gkey;
      unsigned mb = __ballot_sync(0xffffffffu, mem);
      sb &= ~mb;
      float v[32];
#pragma unroll
      for (int s = 0; s < 12; s++) v[s] = mem ? J1[s] + J2[s] : 0.f;
#pragma unroll
      for (int s = 0; s < 8; s++) v[12 + s] = mem ? R[s] : 0.f;
#pragma unroll
      for (int s = 20; s < 32; s++) v[s] = 0.f;
      float sum = transpose_reduce(v, lane);
      if (mem) done = true;
      if (lane < 20) {
        int gi, gj, gk;
        unpack(g, gkey, gi, gj, gk);
        int comp, di, dj, dk;
        slot_offset(lane, comp, di, dj, dk);
        bool ib_ok = in_box(bx, gi, gj, gk);
        deposit_one(a, bx, box, comp, gi + di, gj + dj, gk + dk, to_fix(sum, a.qfix), ib_ok);
      }
    }
    // lanes left: per-lane deposits (cell changed, boundary event, or a
    // third cell in the warp)
    if (live && (!done || !simple)) {
      if (simple) {
        bool ok = in_box(bx, ib, jb, kb);
#pragma unroll
        for (int s = 0; s < 20; s++) {
          int comp, di, dj, dk;
          slot_offset(s, comp, di, dj, dk);
          float val = s < 12 ? J1[s] + J2[s] : R[s - 12];
          deposit_one(a, bx, box, comp, ib + di, jb + dj, kb + dk, to_fix(val, a.qfix), ok);
        }
      } else {
        bool ok1 = in_box(bx, ib, jb, kb);
        bool ok2 = in_box(bx, ax.ia, ay.ia, az.ia);
#pragma unroll
        for (int s = 0; s < 12; s++) {
          int comp, di, dj, dk;
          slot_offset(s, comp, di, dj, dk);
          deposit_one(a, bx, box, comp, ib + di, jb + dj, kb + dk, to_fix(J1[s], a.qfix), ok1);
          deposit_one(a, bx, box, comp, ax.ia + di, ay.ia + dj, az.ia + dk, to_fix(J2[s], a.qfix), ok2);
        }
        if (!dead) {
          bool ok3 = in_box(bx, ax.nc, ay.nc, az.nc);
#pragma unroll
          for (int s = 0; s < 8; s++) {
            int comp, di, dj, dk;
            slot_offset(12 + s, comp, di, dj, dk);
            deposit_one(a, bx, box, comp, ax.nc + di, ay.nc + dj, az.nc + dk, to_fix(R[s], a.qfix), ok3);
          }
        }
      }
    }
  }
  __syncthreads();
  // flush the tile accumulator into the global int64 arrays
  for (int e = threadIdx.x; e < nbox; e += blockDim.x) {
    unsigned long long v = box[e];
    if (v == 0ull) continue;
    int li = e % bx.B, lj = (e / bx.B) % bx.B, lk = (e / (bx.B * bx.B)) % bx.B, comp = e / (bx.B * bx.B * bx.B);
    int i = bx.o[0] + li, j = bx.o[1] + lj, k = bx.o[2] + lk;
    if (comp == 0) {
      if (i < -1 || j < -1 || k < -1 || i > g.nx + 1 || j > g.ny + 1 || k > g.nz + 1) {
        report_bad(a.status, a.diag, SITE_FX_FLUSH, t, i + 100000LL * j + 10000000000LL * k);
        continue;
      }
      atomicAdd(&a.acc_rho[a.fr.at(0, i, j, k)], v);
    } else {
      if (i < -4 || j < -4 || k < -4 || i > g.nx + 4 || j > g.ny + 4 || k > g.nz + 4) {
        report_bad(a.status, a.diag, SITE_FX_FLUSH, t, i + 100000LL * j + 10000000000LL * k);
        continue;
      }
      atomicAdd(&a.acc_j[a.fj.at(comp - 1, i, j, k)], v);
    }
  }
}

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
  for (int d = 0; d < 3; d++) f.bits[d] = ceil_log2(n[d]);
  if (f.bits[0] + f.bits[1] + f.bits[2] > 31)
    return set_error(ctx, EMSESG_ERR_ARG, "grid needs more than 31 bits of packed cell index");
  for (int d = 0; d < 3; d++) {
    int t = c.sort_tile[d] > 0 ? c.sort_tile[d] : 8;
    f.tile[d] = std::min(t, n[d]);
    f.ntile[d] = (n[d] + f.tile[d] - 1) / f.tile[d];
  }
  int tmax = std::max(f.tile[0], std::max(f.tile[1], f.tile[2]));
  if (tmax > 16) return set_error(ctx, EMSESG_ERR_ARG, "FP32 form tiles are at most 16 cells per axis");
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
  int B = tmax + 2 * GUARD + 1;
  int smem = 4 * B * B * B * (int)sizeof(unsigned long long);
  EMSESG_CUDA(ctx, cudaFuncSetAttribute(k_fx_push, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
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
  int B = tmax + 2 * GUARD + 1;
  int smem = 4 * B * B * B * (int)sizeof(unsigned long long);
  for (int is = 0; is < c.nspec; is++) {
    if (ctx->totalp[is] == 0) continue;
    FxPushArgs a{};
    int64_t off = ctx->seg.base[is];
    a.pos = f.pos + off; a.vx = f.vx + off; a.vy = f.vy + off; a.vz = f.vz + off;
    a.tile_start = f.tile_start + (int64_t)is * (f.ntiles + 1);
    a.f0 = f.fnode; a.f1 = f.fnode2;
    a.acc_rho = acc_rho; a.acc_j = acc_j;
    a.fr = fr; a.fj = fj;
    a.g = g;
    for (int d = 0; d < 3; d++) a.npbnd[d] = c.npbnd[is][d];
    double gustep = ustep;
    a.gustep = (float)gustep;
    a.qmp = (float)(c.qm[is] * gustep * 0.5);
    a.rustep = (float)(1.0 / ustep);
    a.qfix = (float)(c.q[is] * 1099511627776.0);
    a.nesc = &ctx->d_counter->nesc[is];
    a.status = ctx->d_status;
    a.diag = ctx->d_diag;
    EMSESG_LAUNCH(ctx, "fx_push", k_fx_push, (unsigned)f.ntiles, FX_THREADS, smem, a);
  }
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
