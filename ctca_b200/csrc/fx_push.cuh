// fx_push.cuh -- the fused push + zigzag current + CIC charge kernel of the
// FP32 / fixed-point form (included by fx.cu inside its private namespace).
//
// Layout.  The sort leaves every (species, cell tile) in a padded region of
// L rows x PUSH_THREADS slots, thread-major: the particle of sorted rank q in
// the tile sits in row q % L, column q / L.  Column t of the region is thus
// thread t's contiguous run of the cell-sorted order, and row r is one
// coalesced stretch of PUSH_THREADS records.  Empty slots hold DEAD cells.
//
// One CTA pushes one region with 736 threads; a 24th warp streams the rows
// into a 3-stage shared-memory ring with cp.async.bulk (TMA 1-D copies
// completing on mbarriers) and never computes, so a warp busy with its
// queues never holds up the stream; pushing warps release a stage through an
// "empty" mbarrier once they hold their particle.  The
// tile's FP32 E/B nodes (tile + 1-cell guard) sit in shared memory.
//
// Per particle: trilinear gather, Buneman-Boris, move.  A particle that
// stays inside its cell (the common case) adds its two zigzag segments and
// its CIC charge to 20 FP32 registers that follow the thread's current cell
// ("run"); when the run's cell changes the 20 sums go through a per-warp
// queue and are added, converted to int64 fixed point, into the CTA's tile
// accumulator by all lanes together.  A particle that stays in its cell
// but is out of place in the thread's run (it changed cell since the sort)
// puts its 20 values into the same queue as a one-particle run.  A particle
// that leaves its cell (or whose cell lies outside the tile box) is appended
// to a per-warp "cross" queue; when 32 are queued, every lane takes one and
// runs the general path (per-axis boundary rules, relay point, two segments
// in different cells, charge at the new cell) with direct int64 atomics.  So
// the divergent work of the few cell-crossing particles runs with all lanes
// busy.
//
// Determinism: a run's FP32 partial sums follow the thread's fixed order;
// every conversion to fixed point is of one value; integer atomics commute.
// Two runs on the same input give the same bits.

// 23 pushing warps + 1 streaming warp: 24 warps, 6 on each SM sub-partition,
// at 80 registers a thread (a few values spill).  The kernel is bound by
// latency more than by issue or memory: at 128^3 x 64 ppc it pushed in
// 8.16 ms with 480-slot rows (16 warps, 128 registers), 7.53 with 608 (20
// warps, 96 registers), 7.20 with 736.
constexpr int PUSH_THREADS = 736;           // pushing threads = slots per row
constexpr int PUSH_WARPS = PUSH_THREADS / 32;
constexpr int PUSH_BLOCK = PUSH_THREADS + 32;  // + one warp that streams the rows
constexpr int PG = 1;           // guard cells around the tile
constexpr int NSTAGE = 3;       // row ring stages (up to NSTAGE - 1 rows in flight)
// Stages of the push's ring: the charge-only push (no current) has the
// shared memory for one more.
__host__ __device__ constexpr int push_stages(bool jd) { return jd ? NSTAGE : NSTAGE + 1; }
constexpr int NJ = 12;          // zigzag node values of one cell
constexpr int NR = 8;           // CIC node values of one cell
constexpr int RQW = NJ + NR + 1;  // run-queue entry: 20 sums + box index of the cell (charge only: 8 + 1)
constexpr int RQ_DRAIN = 8;     // drain the run queue at this many entries
constexpr int RQCAP = RQ_DRAIN + 32;
constexpr int XQW = 8;          // general-path entry: slot, cell, 3 offsets, 3 velocities
constexpr int XLCAP = 128;      // per-warp list of cross slots (emptied when nearly full)
constexpr uint32_t ROW_BYTES = PUSH_THREADS * (16 + 3 * 4);
static_assert(PUSH_THREADS == EMSESG_FX_ROW_SLOTS, "row width of the thread-major layout");
static_assert(ROW_BYTES % 16 == 0 && (PUSH_THREADS * 4) % 16 == 0, "bulk copies move whole 16-byte units");

// Bodies of the FP32 form, in the order of cfg.body.  Box bodies (geotype
// 0/1 with integer bounds): the absorption test and the per-surface-cell
// counts; faces -x,+x,-y,+y,-z,+z, a face's cells with its first tangential
// axis fastest (x faces: y then z; y faces: x then z; z faces: x then y).
// Cylinders (geotype 2) and spheres (3): the absorption test of the end
// point (psolve1.F90:684-712) and the body's influx; lo / hi are then the
// cells their bounding box touches, and they have no surface cells.
struct Bodies {
  int n;                        // bodies
  int ipc[EMSESG_INPC];         // their index in cfg.body
  int kind[EMSESG_INPC];        // 0 box, 2 cylinder, 3 sphere
  int lo[EMSESG_INPC][3], hi[EMSESG_INPC][3];
  int64_t off[EMSESG_INPC][6];  // first surface cell of each face (boxes)
  int64_t nsurf;                // surface cells of all box bodies
  int ncurved;                  // cylinders and spheres
  int cax[EMSESG_INPC];         // cylinder axis 0..2; its transverse axes are cax+1, cax+2 (mod 3)
  float cen[EMSESG_INPC][3];    // sphere centre; cylinder: cyl_axis(1:2) in [cax+1], [cax+2]
  float edge[EMSESG_INPC][2];   // cylinder extent along its axis (inclusive)
  float r2[EMSESG_INPC];        // radius squared (strict inside)
};

// Whether the point (cell ac, offset af per axis) lies inside curved body q
// (psolve1.F90:684-712: d1^2 + d2^2 < r^2 with the axial coordinate within
// the cylinder's edges, inclusive; |x - c|^2 < r^2 for a sphere).  Each
// difference is taken from the integer cell first, so it keeps the offset's
// precision.
__device__ __forceinline__ bool in_curved(const Bodies& bd, int q, const int (&ac)[3], const float (&af)[3]) {
  if (bd.kind[q] == 3) {
    float s = 0.f;
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const float x = ((float)ac[d] - bd.cen[q][d]) + af[d];
      s = fmaf(x, x, s);
    }
    return s < bd.r2[q];
  }
  const int c0 = bd.cax[q], c1 = c0 == 2 ? 0 : c0 + 1, c2 = c0 == 0 ? 2 : c0 - 1;
  const float xl = ((float)ac[c0] - bd.edge[q][0]) + af[c0];
  const float xu = ((float)ac[c0] - bd.edge[q][1]) + af[c0];
  if (!(xl >= 0.f && xu <= 0.f)) return false;
  const float d1 = ((float)ac[c1] - bd.cen[q][c1]) + af[c1];
  const float d2 = ((float)ac[c2] - bd.cen[q][c2]) + af[c2];
  return fmaf(d1, d1, d2 * d2) < bd.r2[q];
}

// Slab mode (the grid is one z slab of a larger grid, periodic in z, cut
// into slabs of equal thickness): particles that leave through a z face go
// to the neighbouring slab's rank.  Their records, in that rank's frame (the
// periodic wrap of this slab), per species and direction: region
// (2 is + dir) of cap records, dir 0 through z = 0, 1 through z = nz.  pid
// holds the particle's slot here (the order of the records is then made
// independent of the atomics).
struct Outbox {
  emsesg_particle* rec;         // null: not in slab mode
  unsigned long long* count;    // [2 nspec]
  int64_t cap;
};

struct FxPushArgs {
  float4* pos;                  // all species regions (the step's result)
  float* vx;
  float* vy;
  float* vz;
  const float4* rpos;           // the state read (the same arrays, or for a
  const float* rvx;             // move-only step, those of a kept copy)
  const float* rvy;
  const float* rvz;
  const int64_t* tile_start;    // [nspec][ntiles+1] sorted ranks (live particles)
  const int64_t* tile_pad;      // [nspec][ntiles+1] slot offsets of the padded regions
  const int64_t* chunk_start;   // [nspec][ntiles+1] first CTA (row chunk) of each tile
  int64_t off[EMSESG_ISPEC];    // region base per species
  int npbnd[EMSESG_ISPEC][3];
  float qmp[EMSESG_ISPEC], qfix[EMSESG_ISPEC];
  float gustep, rustep;
  const float4* __restrict__ f0;
  const float4* __restrict__ f1;
  unsigned long long* acc_rho;  // rho layout (1, -1:n+1)
  unsigned long long* acc_j;    // aj layout (3, -4:n+4)
  FieldDesc fr, fj;
  Geo g;
  int64_t ntiles;
  int chunk_rows;               // rows of a tile region per CTA
  int* nesc;                    // counter nesc(is), one int per species
  emsesg_counter* gc;           // influx / infhist of the body absorption
  unsigned long long* surf;     // [nspec][nsurf] absorbed - emitted counts
  Bodies bd;
  Outbox ob;
  int* status;
  long long* diag;
  // the tiles of this launch: t_lo .. t_lo + t_n - 1 (t_n = 0: every tile;
  // a step whose eb arrives in z chunks pushes its tile layers in parts)
  int64_t t_lo, t_n;
  // a part (PARTS) holds the node planes 0..zready; it marks here (one bit
  // per slot) a particle that would gather from a higher plane, which
  // k_fx_deferred pushes after the last part
  int zready;
  uint32_t* defer;
};

// ---------------------------------------------------------------- PTX
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(smem_u32(b)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
// Bounded wait: gives up after about one second.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity) {
  if (mbar_try_wait(b, parity)) return true;
  const uint64_t t0 = global_ns();
  for (uint32_t it = 0;; it++) {
    if (mbar_try_wait(b, parity)) return true;
    if ((it & 255u) == 255u && global_ns() - t0 > 1000000000ull) return false;
  }
}
// 1-D bulk copy global -> shared, completing on an mbarrier (both addresses
// 16-byte aligned, size a multiple of 16).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// ---------------------------------------------------------------- moves
// Per-axis move and outer boundary of psolve1.F90:366-606 on (cell, offset)
// pairs.  In: cell ib, offset ob, displacement d.  Out: the "after" point
// xlocala = (ac, af), its cell ia, the relay point xr = (rc, rf), the stored
// new position (nc, nf), and flags.
struct Axis {
  int ac, ia, rc, nc;
  float af, rf, nf;
  bool dead, flip, crossed;
};

// The outer boundary rules for an "after" cell ac outside 0..n-1.
__device__ __forceinline__ Axis axis_boundary(int ib, float ob, int ac, float af, int n, int npbnd) {
  Axis o;
  o.dead = false;
  o.flip = false;
  o.crossed = true;
  if (ac < 0) {  // p%x < 0
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
  } else {  // p%x >= slx
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
  }
  return o;
}

__device__ __forceinline__ Axis axis_move(int ib, float ob, float d, int n, int npbnd) {
  const float s = ob + d;
  const float fl = floorf(s);
  int ac = ib + (int)fl;
  float af = s - fl;
  if (af >= 1.0f) { af = 0.0f; ac += 1; }
  if ((unsigned)ac >= (unsigned)n) return axis_boundary(ib, ob, ac, af, n, npbnd);
  Axis o;
  o.dead = false;
  o.flip = false;
  o.crossed = false;
  o.ac = ac; o.af = af; o.ia = ac; o.nc = ac; o.nf = af;
  const bool same = ac == ib;
  o.rc = same ? ib : max(ib, ac);
  o.rf = same ? (ob + af) * 0.5f : 0.f;
  return o;
}

// Node offsets of the 12 zigzag values of a cell: 0-3 JX at (0,a,b), 4-7 JY
// at (a,0,b), 8-11 JZ at (a,b,0) with (a,b) = (s&1, s>>1&1), in the order of
// the scatter-adds of psolve1.F90:759-789 (w1, w2, w3, w4 per component).
__host__ __device__ constexpr int jcomp(int s) { return 1 + (s >> 2); }
__host__ __device__ constexpr int jdi(int s) { return s < 4 ? 0 : (s & 1); }
__host__ __device__ constexpr int jdj(int s) { return s < 4 ? (s & 1) : (s < 8 ? 0 : ((s >> 1) & 1)); }
__host__ __device__ constexpr int jdk(int s) { return s < 8 ? ((s >> 1) & 1) : 0; }
// CIC corners v1..v8 (charge.F90:202-209): (0,0,1) (1,0,1) (1,1,1) (0,1,1)
// (0,0,0) (1,0,0) (1,1,0) (0,1,0).
__host__ __device__ constexpr int rdi(int r) { return ((r & 3) == 1 || (r & 3) == 2) ? 1 : 0; }
__host__ __device__ constexpr int rdj(int r) { return (r & 3) >= 2 ? 1 : 0; }
__host__ __device__ constexpr int rdk(int r) { return r < 4 ? 1 : 0; }

template <int B>
struct BoxT {
  static constexpr int B2 = B * B;
  static constexpr int B3 = B * B * B;
  __host__ __device__ static constexpr int joff(int s) { return jcomp(s) * B3 + jdk(s) * B2 + jdj(s) * B + jdi(s); }
  __host__ __device__ static constexpr int roff(int r) { return rdk(r) * B2 + rdj(r) * B + rdi(r); }
};

__device__ __forceinline__ long long to_fix(float v, float scale) { return __float2ll_rn(v * scale); }

// Adds v to a 64-bit accumulator in shared memory with 32-bit atomics (a
// 64-bit shared-memory atomic add is much slower): the low word first, its
// carry out then goes with the high word.  The carries counted by all
// additions add up to the wraps of the low word, so the final value is the
// 64-bit sum in any order; only the final value is read.
__device__ __forceinline__ void box_add(unsigned long long* p, unsigned long long v) {
  unsigned int* w = reinterpret_cast<unsigned int*>(p);  // little-endian: low word first
  const unsigned int lo = (unsigned int)v, hi = (unsigned int)(v >> 32);
  const unsigned int old = atomicAdd(w, lo);
  const unsigned int h = hi + (old + lo < old ? 1u : 0u);
  if (h) atomicAdd(w + 1, h);
}

// Global arrays for deposits whose cell lies outside the tile box.
struct Sink {
  unsigned long long* acc_rho;
  unsigned long long* acc_j;
  FieldDesc fr, fj;
  int nx, ny, nz;
  int* status;
  long long* diag;
};

// Box index of cell (i,j,k) when its 2x2x2 node block lies inside the box,
// else -1.
template <int B>
__device__ __forceinline__ int box_base(const int (&o)[3], int i, int j, int k) {
  int li = i - o[0], lj = j - o[1], lk = k - o[2];
  bool ok = (unsigned)li < (unsigned)(B - 1) && (unsigned)lj < (unsigned)(B - 1) && (unsigned)lk < (unsigned)(B - 1);
  return ok ? (lk * B + lj) * B + li : -1;
}

struct V12 { float v[NJ]; };
struct V8 { float v[NR]; };

// Node sets whose cell lies outside the box: global int64 atomics with
// bounds checks (rare; the values come by value so that the callers'
// register arrays keep no address).
__device__ __forceinline__ void put_j_global(Sink s, int i, int j, int k, V12 v, float qfix) {
  for (int q = 0; q < NJ; q++) {
    const long long f = to_fix(v.v[q], qfix);
    if (f == 0) continue;
    const int ii = i + jdi(q), jj = j + jdj(q), kk = k + jdk(q);
    if (ii < -4 || jj < -4 || kk < -4 || ii > s.nx + 4 || jj > s.ny + 4 || kk > s.nz + 4) {
      report_bad(s.status, s.diag, SITE_FX_DEPOSIT, -2, ii + 100000LL * jj + 10000000000LL * kk);
      continue;
    }
    atomicAdd(&s.acc_j[s.fj.at(jcomp(q) - 1, ii, jj, kk)], (unsigned long long)f);
  }
}

__device__ __forceinline__ void put_r_global(Sink s, int i, int j, int k, V8 v, float qfix) {
  for (int r = 0; r < NR; r++) {
    const long long f = to_fix(v.v[r], qfix);
    if (f == 0) continue;
    const int ii = i + rdi(r), jj = j + rdj(r), kk = k + rdk(r);
    if (ii < -1 || jj < -1 || kk < -1 || ii > s.nx + 1 || jj > s.ny + 1 || kk > s.nz + 1) {
      report_bad(s.status, s.diag, SITE_FX_DEPOSIT, -1, ii + 100000LL * jj + 10000000000LL * kk);
      continue;
    }
    atomicAdd(&s.acc_rho[s.fr.at(0, ii, jj, kk)], (unsigned long long)f);
  }
}

// One zigzag node set (12 values) of cell (i,j,k): into the box, or into the
// global arrays when the cell lies outside the box.
template <int B>
__device__ __forceinline__ void put_j(unsigned long long* box, const int (&o)[3], const Sink& s, int i, int j, int k,
                                      const float (&v)[NJ], float qfix) {
  const int base = box_base<B>(o, i, j, k);
  if (base >= 0) {
#pragma unroll
    for (int q = 0; q < NJ; q++) box_add(&box[base + BoxT<B>::joff(q)], (unsigned long long)to_fix(v[q], qfix));
  } else {
    V12 w;
#pragma unroll
    for (int q = 0; q < NJ; q++) w.v[q] = v[q];
    put_j_global(s, i, j, k, w, qfix);
  }
}

template <int B>
__device__ __forceinline__ void put_r(unsigned long long* box, const int (&o)[3], const Sink& s, int i, int j, int k,
                                      const float (&v)[NR], float qfix) {
  const int base = box_base<B>(o, i, j, k);
  if (base >= 0) {
#pragma unroll
    for (int r = 0; r < NR; r++) box_add(&box[base + BoxT<B>::roff(r)], (unsigned long long)to_fix(v[r], qfix));
  } else {
    V8 w;
#pragma unroll
    for (int r = 0; r < NR; r++) w.v[r] = v[r];
    put_r_global(s, i, j, k, w, qfix);
  }
}

template <bool SMEM>
__device__ __forceinline__ void gather8(const float4* f0, const void* f1v, int64_t n5, int64_t sy, int64_t sz,
                                        const float (&w)[8], float (&e)[3], float (&b)[3]) {
  const int64_t idx[8] = {n5 + sz, n5 + sz + 1, n5 + sz + 1 + sy, n5 + sz + sy, n5, n5 + 1, n5 + 1 + sy, n5 + sy};
  float ex = 0.f, ey = 0.f, ez = 0.f, bx = 0.f, by = 0.f, bz = 0.f;
#pragma unroll
  for (int c = 0; c < 8; c++) {
    float4 p;
    float2 q;
    if (SMEM) {
      p = f0[idx[c]];
      q = reinterpret_cast<const float2*>(f1v)[idx[c]];
    } else {
      p = __ldg(&f0[idx[c]]);
      float4 q4 = __ldg(&reinterpret_cast<const float4*>(f1v)[idx[c]]);
      q = make_float2(q4.x, q4.y);
    }
    ex += p.x * w[c];
    ey += p.y * w[c];
    ez += p.z * w[c];
    bx += p.w * w[c];
    by += q.x * w[c];
    bz += q.y * w[c];
  }
  e[0] = ex; e[1] = ey; e[2] = ez;
  b[0] = bx; b[1] = by; b[2] = bz;
}

// The same gather from the tile's shared-memory nodes (box index `base`,
// compile-time strides).
template <int B>
__device__ __forceinline__ void gather8_smem(const float4* f0, const float2* f1, int base, const float (&w)[8],
                                             float (&e)[3], float (&b)[3]) {
  constexpr int SY = B, SZ = B * B;
  constexpr int off[8] = {SZ, SZ + 1, SZ + 1 + SY, SZ + SY, 0, 1, 1 + SY, SY};
  float ex = 0.f, ey = 0.f, ez = 0.f, bx = 0.f, by = 0.f, bz = 0.f;
#pragma unroll
  for (int c = 0; c < 8; c++) {
    const float4 p = f0[base + off[c]];
    const float2 q = f1[base + off[c]];
    ex += p.x * w[c];
    ey += p.y * w[c];
    ez += p.z * w[c];
    bx += p.w * w[c];
    by += q.x * w[c];
    bz += q.y * w[c];
  }
  e[0] = ex; e[1] = ey; e[2] = ez;
  b[0] = bx; b[1] = by; b[2] = bz;
}

// Trilinear gather of E and B at the particle (from the tile's shared nodes
// when its cell lies in the box, gb >= 0, else from the global node field)
// and the Buneman-Boris velocity update (psolve1.F90:186-272).  The shared
// nodes hold the fields already multiplied by the species' qmp; the global
// ones are multiplied here.
template <int B>
__device__ __forceinline__ void kick(const FxPushArgs& a, const float4* sf0, const float2* sf1, int gb, int ib, int jb,
                                     int kb, const float4& ps, float qmp, float& vx, float& vy, float& vz) {
  const float x1 = ps.x, y1 = ps.y, z1 = ps.z;
  const float xy1 = x1 * y1, xz1 = x1 * z1, yz1 = y1 * z1, z2 = 1.0f - z1;
  const float xz2 = x1 * z2, yz2 = y1 * z2;
  float wv[8];
  wv[2] = xy1 * z1; wv[1] = xz1 - wv[2]; wv[3] = yz1 - wv[2]; wv[0] = z1 - xz1 - wv[3];
  wv[6] = xy1 * z2; wv[5] = xz2 - wv[6]; wv[7] = yz2 - wv[6]; wv[4] = z2 - xz2 - wv[7];
  float fe[3], fb[3];
  if (gb >= 0) {
    gather8_smem<B>(sf0, sf1, gb, wv, fe, fb);
  } else {
    const int64_t sy = a.g.nx + 1, sz = (int64_t)(a.g.nx + 1) * (a.g.ny + 1);
    gather8<false>(a.f0, a.f1, ib + sy * jb + sz * kb, sy, sz, wv, fe, fb);
#pragma unroll
    for (int d = 0; d < 3; d++) {
      fe[d] *= qmp;
      fb[d] *= qmp;
    }
  }
  const float eex = fe[0], eey = fe[1], eez = fe[2];
  const float bbx = fb[0], bby = fb[1], bbz = fb[2];
  const float boris = __fdividef(2.0f, 1.0f + bbx * bbx + bby * bby + bbz * bbz);
  vx += eex; vy += eey; vz += eez;
  const float vxt = vx + vy * bbz - vz * bby;
  const float vyt = vy + vz * bbx - vx * bbz;
  const float vzt = vz + vx * bby - vy * bbx;
  vx += boris * (vyt * bbz - vzt * bby);
  vy += boris * (vzt * bbx - vxt * bbz);
  vz += boris * (vxt * bby - vyt * bbx);
  vx += eex; vy += eey; vz += eez;
}

// Empties a warp's run queue.  The queue's (entry, slot) items are dealt
// out to the lanes in order, item m to lane m mod 32, so every pass keeps all
// 32 lanes busy however few entries are queued; the items of one entry go
// to 20 different nodes.  An entry holds its 20 sums and the box index of
// its cell (only cells inside the box are queued).
template <int NC>
__device__ __forceinline__ void drain_runs(unsigned long long* box, const int* slot_off, const float* q, int qn,
                                           float qfix, int lane) {
  static_assert(NC > 0 && NC <= 32, "an entry's sums fit one pass");
  constexpr int QW = NC + 1;
  __syncwarp();
  const int items = qn * NC;
  int e = lane / NC, sl = lane % NC;
  for (int m = lane; m < items; m += 32) {
    const float* en = q + e * QW;
    const int base = __float_as_int(en[NC]);
    const long long f = to_fix(en[sl], qfix);
    if (f) box_add(&box[base + slot_off[sl]], (unsigned long long)f);
    // m += 32: 32 = (32 / NC) * NC + 32 % NC
    sl += 32 % NC;
    e += 32 / NC;
    if (sl >= NC) {
      sl -= NC;
      e += 1;
    }
  }
  __syncwarp();
}

struct CrossCtx {
  float4* gpos;                 // the tile region's first slot
  float* gvx;
  float* gvy;
  float* gvz;
  float gustep, rustep, qfix;
  int nb[3];
  const Bodies* bd;
  emsesg_counter* gc;
  unsigned long long* surf;     // this species' surface counts
  int is;
  int64_t slot_base;            // slot of gpos[0] in the particle arrays
  const Outbox* ob;
  int* status;
};

// Absorption of the end point by the bodies in their order, the first that
// holds it taking it (psolve1.F90:639-715).  A box tests a = (ac, af) per
// axis (:644-662, inclusive bounds) and counts influx, infhist and the
// surface cell of the face crossed last on the way from b = (ib, ob) (the
// rule of the oracle's orc_surface_cell); a cylinder or sphere tests the
// stored position (nc, nf) and counts influx and infhist.  Returns 0 (not
// absorbed), ABS_BOX (the particle stops at the relay point: no second
// zigzag segment, :660-662) or ABS_CURVED (both segments deposited).
constexpr int ABS_BOX = 1, ABS_CURVED = 2;
template <bool CURV>
__device__ __forceinline__ int body_absorb(const CrossCtx& c, const int (&ib)[3], const float (&ob)[3],
                                           const Axis* a3) {
  const Bodies& bd = *c.bd;
  for (int q = 0; q < bd.n; q++) {
    if (CURV && bd.kind[q] != 0) {
      const int nc3[3] = {a3[0].nc, a3[1].nc, a3[2].nc};
      const float nf3[3] = {a3[0].nf, a3[1].nf, a3[2].nf};
      if (!in_curved(bd, q, nc3, nf3)) continue;
      atomicAdd(&c.gc->influx[c.is][bd.ipc[q]], 1);
      atomicAdd(&c.gc->infhist[c.is][bd.ipc[q]][0], 1);
      return ABS_CURVED;
    }
    bool in = true;
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const int ac = a3[d].ac;
      in = in && ac >= bd.lo[q][d] && (ac < bd.hi[q][d] || (ac == bd.hi[q][d] && a3[d].af == 0.0f));
    }
    if (!in) continue;
    const int ipc = bd.ipc[q];
    atomicAdd(&c.gc->influx[c.is][ipc], 1);
    atomicAdd(&c.gc->infhist[c.is][ipc][0], 1);
    // face crossed last: the largest entry time along b -> a
    int best = -1, side = 0;
    float tb = -1.0f;
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const int lo = bd.lo[q][d], hi = bd.hi[q][d];
      const float den = (float)(a3[d].ac - ib[d]) + (a3[d].af - ob[d]);
      float t = -1.0f;
      int sd = 0;
      if (ib[d] < lo) { t = ((float)(lo - ib[d]) - ob[d]) / den; sd = 0; }
      else if (ib[d] > hi || (ib[d] == hi && ob[d] > 0.0f)) { t = ((float)(hi - ib[d]) - ob[d]) / den; sd = 1; }
      if (t > tb) { tb = t; best = d; side = sd; }
    }
    if (best < 0) {  // start point inside: the nearest face of the end point
      float dm = 3.0e38f;
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const float x = (float)a3[d].ac + a3[d].af;
        if (x - (float)bd.lo[q][d] < dm) { dm = x - (float)bd.lo[q][d]; best = d; side = 0; }
        if ((float)bd.hi[q][d] - x < dm) { dm = (float)bd.hi[q][d] - x; best = d; side = 1; }
      }
    }
    const int e1 = best == 0 ? 1 : 0, e2 = best == 2 ? 1 : 2;
    const int c1 = best == 0 ? a3[1].ac : a3[0].ac;  // selects keep a3 in registers
    const int c2 = best == 2 ? a3[1].ac : a3[2].ac;
    const int u = min(max(c1, bd.lo[q][e1]), bd.hi[q][e1] - 1) - bd.lo[q][e1];
    const int v = min(max(c2, bd.lo[q][e2]), bd.hi[q][e2] - 1) - bd.lo[q][e2];
    const int64_t cellx = bd.off[q][2 * best + side] + u + (int64_t)(bd.hi[q][e1] - bd.lo[q][e1]) * v;
    atomicAdd(&c.surf[cellx], 1ull);
    return ABS_BOX;
  }
  return 0;
}

// General path for one particle that left its cell (or whose cell lies
// outside the box): boundary rules, zigzag with relay point, charge at the
// stored cell; the final record is written here.  CURV = false: no
// cylinder or sphere to test.  JD = false: charge only (no zigzag current).
template <int B, bool DEP = true, bool CURV = true, bool JD = true>
__device__ __forceinline__ int cross_one(const Geo& g, unsigned long long* box, const int (&o)[3], const Sink& sk,
                                         const CrossCtx& c, const float* en) {
  const int loc = __float_as_int(en[0]);
  const uint32_t cell = (uint32_t)__float_as_int(en[1]);
  const float bx = en[2], by = en[3], bz = en[4];
  float vx = en[5], vy = en[6], vz = en[7];
  int ib, jb, kb;
  unpack(g, cell, ib, jb, kb);
  Axis ax = axis_move(ib, bx, vx * c.gustep, g.nx, c.nb[0]);
  Axis ay = axis_move(jb, by, vy * c.gustep, g.ny, c.nb[1]);
  Axis az = axis_move(kb, bz, vz * c.gustep, g.nz, c.nb[2]);
  if (ax.flip) vx = -vx;
  if (ay.flip) vy = -vy;
  if (az.flip) vz = -vz;
  const bool escaped = ax.dead || ay.dead || az.dead;
  int absorbed = 0;
  if (!escaped && c.bd->n > 0) {
    const int ib3[3] = {ib, jb, kb};
    const float ob3[3] = {bx, by, bz};
    const Axis a3[3] = {ax, ay, az};
    absorbed = body_absorb<CURV>(c, ib3, ob3, a3);
  }
  const bool stop = absorbed == ABS_BOX;
  // slab mode: a particle leaving through a z face moves to the neighbouring
  // slab (its stored position, the slab's periodic wrap, is its position
  // there); its current stays here, in the guard planes that the ranks
  // exchange and fold, and its charge is deposited by the receiver
  const bool migrant = c.ob != nullptr && az.crossed && !escaped && !absorbed;
  if (migrant) {
    const int dir = az.ac < 0 ? 0 : 1;
    const unsigned long long q = atomicAdd(&c.ob->count[2 * c.is + dir], 1ull);
    if (q < (unsigned long long)c.ob->cap) {
      emsesg_particle r;
      r.x = (double)ax.nc + (double)ax.nf;
      r.y = (double)ay.nc + (double)ay.nf;
      r.z = (double)az.nc + (double)az.nf;
      r.vx = vx; r.vy = vy; r.vz = vz;
      r.pid = (int32_t)(c.slot_base + loc);
      r.preside = 0; r.nid = 0; r.spec = c.is + 1;
      c.ob->rec[(int64_t)(2 * c.is + dir) * c.ob->cap + (int64_t)q] = r;
    } else {
      atomicOr(c.status, ST_OVERFLOW);
    }
  }
  const bool dead = escaped || absorbed || migrant;
  const uint32_t nc = dead ? DEAD : pack(g, ax.nc, ay.nc, az.nc);
  c.gpos[loc] = make_float4(ax.nf, ay.nf, az.nf, __int_as_float((int)nc));
  c.gvx[loc] = vx;
  c.gvy[loc] = vy;
  c.gvz[loc] = vz;
  if (!DEP) return escaped ? 1 : 0;
  if (JD) {
  // zigzag (psolve1.F90:717-757), integer parts first
  float J[NJ];
  {
    float xd = ((float)(ax.rc - ib) + ax.rf + bx) * 0.5f;
    float yd = ((float)(ay.rc - jb) + ay.rf + by) * 0.5f;
    float zd = ((float)(az.rc - kb) + az.rf + bz) * 0.5f;
    float vvx = ((float)(ax.rc - ib) + (ax.rf - bx)) * c.rustep;
    float vvy = ((float)(ay.rc - jb) + (ay.rf - by)) * c.rustep;
    float vvz = ((float)(az.rc - kb) + (az.rf - bz)) * c.rustep;
    float w;
    w = yd * zd; J[3] = vvx * w; J[1] = vvx * (yd - w); J[2] = vvx * (zd - w); J[0] = vvx * (1.0f - yd - (zd - w));
    w = xd * zd; J[7] = vvy * w; J[5] = vvy * (xd - w); J[6] = vvy * (zd - w); J[4] = vvy * (1.0f - xd - (zd - w));
    w = xd * yd; J[11] = vvz * w; J[9] = vvz * (xd - w); J[10] = vvz * (yd - w); J[8] = vvz * (1.0f - xd - (yd - w));
  }
  // a start point inside a box body moves to the relay point
  // (psolve1.F90:648-651): no first segment
  if (CURV && !escaped) {
    const Bodies& bd = *c.bd;
    const int ib3[3] = {ib, jb, kb};
    const float ob3[3] = {bx, by, bz};
    bool start_in = false;
    for (int q = 0; q < bd.n && !start_in; q++) {
      if (bd.kind[q] != 0) continue;
      bool in = true;
#pragma unroll
      for (int d = 0; d < 3; d++)
        in = in && ib3[d] >= bd.lo[q][d] && (ib3[d] < bd.hi[q][d] || (ib3[d] == bd.hi[q][d] && ob3[d] == 0.0f));
      start_in = in;
    }
    if (start_in) {
#pragma unroll
      for (int q = 0; q < NJ; q++) J[q] = 0.f;
    }
  }
  // both segments in the cell of the start point (a particle that did not
  // change cell): one set of node values.  A particle absorbed by a box
  // stops at the relay point (psolve1.F90:660-662): no second segment.
  const bool one = !stop && ax.ia == ib && ay.ia == jb && az.ia == kb;
  if (!one) put_j<B>(box, o, sk, ib, jb, kb, J, c.qfix);
  if (!stop) {
    float J2[NJ];
    float xd = ((float)(ax.ac - ax.ia) + ax.af + (float)(ax.rc - ax.ia) + ax.rf) * 0.5f;
    float yd = ((float)(ay.ac - ay.ia) + ay.af + (float)(ay.rc - ay.ia) + ay.rf) * 0.5f;
    float zd = ((float)(az.ac - az.ia) + az.af + (float)(az.rc - az.ia) + az.rf) * 0.5f;
    float vvx = ((float)(ax.ac - ax.rc) + (ax.af - ax.rf)) * c.rustep;
    float vvy = ((float)(ay.ac - ay.rc) + (ay.af - ay.rf)) * c.rustep;
    float vvz = ((float)(az.ac - az.rc) + (az.af - az.rf)) * c.rustep;
    float w;
    w = yd * zd; J2[3] = vvx * w; J2[1] = vvx * (yd - w); J2[2] = vvx * (zd - w); J2[0] = vvx * (1.0f - yd - (zd - w));
    w = xd * zd; J2[7] = vvy * w; J2[5] = vvy * (xd - w); J2[6] = vvy * (zd - w); J2[4] = vvy * (1.0f - xd - (zd - w));
    w = xd * yd; J2[11] = vvz * w; J2[9] = vvz * (xd - w); J2[10] = vvz * (yd - w); J2[8] = vvz * (1.0f - xd - (yd - w));
    if (one) {
#pragma unroll
      for (int q = 0; q < NJ; q++) J2[q] += J[q];
    }
    put_j<B>(box, o, sk, ax.ia, ay.ia, az.ia, J2, c.qfix);
  }
  }  // JD
  if (!dead) {
    // charge.F90:152-210 at the stored (wrapped / reflected) position
    float X = ax.nf, Y = ay.nf, Z = az.nf;
    float XY = X * Y, XZ = X * Z, YZ = Y * Z, Z2 = 1.0f - Z, XZ2 = X * Z2, YZ2 = Y * Z2;
    float R[NR];
    R[2] = XY * Z; R[1] = XZ - R[2]; R[3] = YZ - R[2]; R[0] = Z - XZ - R[3];
    R[6] = XY * Z2; R[5] = XZ2 - R[6]; R[7] = YZ2 - R[6]; R[4] = Z2 - XZ2 - R[7];
    put_r<B>(box, o, sk, ax.nc, ay.nc, az.nc, R, c.qfix);
  }
  return escaped ? 1 : 0;
}

// The particles of a warp's cross list (slots in the tile region, still
// holding their position before this step and the velocity the row loop
// gave them): each lane takes one and runs the general path.  Returns the
// number of this lane's particles that escaped.
template <int B, bool DEP, bool CURV, bool JD>
__device__ __forceinline__ int cross_list(const FxPushArgs& a, int is, int64_t slot0, unsigned long long* box,
                                          const int (&o)[3], const int* xl, int xn, int lane) {
  __syncwarp();
  // the context comes from the kernel parameters here, so that the pushing
  // loop keeps none of it in registers
  const Geo& g = a.g;
  const Sink sk{a.acc_rho, a.acc_j, a.fr, a.fj, g.nx, g.ny, g.nz, a.status, a.diag};
  const CrossCtx c{a.pos + slot0, a.vx + slot0, a.vy + slot0, a.vz + slot0, a.gustep, a.rustep, a.qfix[is],
                   {a.npbnd[is][0], a.npbnd[is][1], a.npbnd[is][2]}, &a.bd, a.gc,
                   a.surf + (int64_t)is * a.bd.nsurf, is, slot0, a.ob.rec ? &a.ob : nullptr, a.status};
  int dead = 0;
  for (int e = lane; e < xn; e += 32) {
    const int loc = xl[e];
    const float4 ps = a.rpos[slot0 + loc];  // the position before the step
    const float vx = c.gvx[loc], vy = c.gvy[loc], vz = c.gvz[loc];
    const float en[XQW] = {__int_as_float(loc), ps.w, ps.x, ps.y, ps.z, vx, vy, vz};
    dead += cross_one<B, DEP, CURV, JD>(g, box, o, sk, c, en);
  }
  __syncwarp();
  return dead;
}

// DEP = false: the move only (positions, velocities, boundary rules; no
// current, no charge), for recomputing particle states.  CURV = true: a
// particle may end inside a body without leaving its cell (cylinders or
// spheres; boxes after a load of particles that start inside one): tile
// regions next to a body push every particle on the general path; without
// that the in-cell test keeps its constant bound.
// JD = false (the electrostatic step, psolve2 + charge):
// the charge only -- runs of 8 CIC sums, an accumulator of rho alone, no
// zigzag current.
template <int T, bool DEP = true, bool CURV = false, bool JD = true, bool PARTS = false>
__global__ void __launch_bounds__(PUSH_BLOCK, 1) k_fx_push(FxPushArgs a) {
  constexpr int B = T + 2 * PG + 1;  // box and field tile edge (nodes)
  constexpr int NC = JD ? NJ + NR : NR;  // sums of a run: zigzag J and CIC rho, or rho alone
  constexpr int RO = JD ? NJ : 0;        // first rho sum
  constexpr int QW = NC + 1;             // run-queue entry: the sums and the cell's box index
  constexpr int NACC = (JD ? 4 : 1) * B * B * B;  // accumulator entries (rho, then Jx, Jy, Jz)
  constexpr int NBOX = (NACC + 1) & ~1;           // their 8-byte words, padded so that the ring after them
                                                  // starts on a 16-byte boundary (bulk copies, float4)
  constexpr int NF = B * B * B;
  constexpr int NS = push_stages(JD);  // row ring stages
  static_assert((NBOX * 8) % 16 == 0 && (NBOX * 8 + NS * ROW_BYTES) % 16 == 0,
                "the row ring and the field tile start on 16-byte boundaries");
  extern __shared__ __align__(128) unsigned long long smem[];
  __shared__ __align__(8) uint64_t full_bar[NS];
  __shared__ __align__(8) uint64_t empty_bar[NS];
  __shared__ int slot_off[NC];
  __shared__ int rows_seen;
  const Geo& g = a.g;
  const int is = blockIdx.y;
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const unsigned lt = (1u << lane) - 1u;

  // this CTA's chunk: tile t, rows r0 .. r0 + L - 1 of its region (a tile of
  // more than CHUNK_ROWS rows is pushed by several CTAs, which add their
  // sums into the same global arrays)
  const int64_t* ts = a.tile_start + (int64_t)is * (a.ntiles + 1);
  const int64_t* cs = a.chunk_start + (int64_t)is * (a.ntiles + 1);
  const int64_t t_end = a.t_n > 0 ? a.t_lo + a.t_n : a.ntiles;
  const int64_t b = cs[a.t_lo] + blockIdx.x;
  if (b >= cs[t_end]) return;
  int64_t tlo = a.t_lo, thi = t_end;  // the last tile with cs[t] <= b
  while (thi - tlo > 1) {
    const int64_t mid = (tlo + thi) >> 1;
    if (cs[mid] <= b) tlo = mid;
    else thi = mid;
  }
  const int t = (int)tlo;
  const int64_t n = ts[t + 1] - ts[t];
  if (n <= 0) return;
  const int r0 = (int)(b - cs[t]) * a.chunk_rows;
  const int L = min((int)((n + PUSH_THREADS - 1) / PUSH_THREADS) - r0, a.chunk_rows);
  if (L <= 0) return;
  const int64_t slot0 = a.off[is] + a.tile_pad[(int64_t)is * (a.ntiles + 1) + t] + (int64_t)r0 * PUSH_THREADS;

  int tx = t % g.nt[0], ty = (t / g.nt[0]) % g.nt[1], tz = t / (g.nt[0] * g.nt[1]);
  const int o[3] = {tx * g.t[0] - PG, ty * g.t[1] - PG, tz * g.t[2] - PG};
  unsigned long long* box = smem;
  float4* stpos = reinterpret_cast<float4*>(smem + NBOX);
  float* stvx = reinterpret_cast<float*>(stpos + NS * PUSH_THREADS);
  float* stvy = stvx + NS * PUSH_THREADS;
  float* stvz = stvy + NS * PUSH_THREADS;
  float4* sf0 = reinterpret_cast<float4*>(stvz + NS * PUSH_THREADS);
  float2* sf1 = reinterpret_cast<float2*>(sf0 + NF);
  float* rq = reinterpret_cast<float*>(sf1 + NF) + warp * RQCAP * QW;
  int* xl = reinterpret_cast<int*>(reinterpret_cast<float*>(sf1 + NF) + PUSH_WARPS * RQCAP * QW) + warp * XLCAP;

  float4* gpos = a.pos + slot0;
  float* gvx = a.vx + slot0;
  float* gvy = a.vy + slot0;
  float* gvz = a.vz + slot0;
  const float4* rgpos = a.rpos + slot0;
  const float* rgvx = a.rvx + slot0;
  const float* rgvy = a.rvy + slot0;
  const float* rgvz = a.rvz + slot0;

  if (tid == 0) {
    for (int s = 0; s < NS; s++) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], PUSH_WARPS);
    }
    mbar_fence_init();
  }
  if (tid < NC) slot_off[tid] = tid < RO ? BoxT<B>::joff(tid) : BoxT<B>::roff(tid - RO);
  if (DEP)
    for (int e = tid; e < NBOX; e += PUSH_BLOCK) box[e] = 0ull;
  const int64_t sy = g.nx + 1, sz = (int64_t)(g.nx + 1) * (g.ny + 1);
  const float sq = a.qmp[is];  // the tile's fields times the species' qmp
  for (int e = tid; e < NF; e += PUSH_BLOCK) {
    int li = e % B, lj = (e / B) % B, lk = e / (B * B);
    int gi = o[0] + li, gj = o[1] + lj, gk = o[2] + lk;
    float4 p = make_float4(0.f, 0.f, 0.f, 0.f), q = p;
    if (gi >= 0 && gj >= 0 && gk >= 0 && gi <= g.nx && gj <= g.ny && gk <= g.nz) {
      int64_t gn = gi + sy * gj + sz * gk;
      p = __ldg(&a.f0[gn]);
      q = __ldg(&a.f1[gn]);
    }
    sf0[e] = make_float4(p.x * sq, p.y * sq, p.z * sq, p.w * sq);
    sf1[e] = make_float2(q.x * sq, q.y * sq);
  }
  __syncthreads();

  int issued = 0;  // rows issued (producer lane 0)
  if (warp == PUSH_WARPS) {
    // Row producer: row r goes to stage r % NS once every pushing warp
    // released the row that used that stage before.
    if (lane == 0) {
      for (int r = 0; r < L; r++) {
        const int s = r % NS;
        if (r >= NS && !mbar_wait(&empty_bar[s], (uint32_t)((r / NS - 1) & 1))) {
          report_bad(a.status, a.diag, SITE_FX_PUSH, -4, t);
          break;
        }
        mbar_expect_tx(&full_bar[s], ROW_BYTES);
        const int64_t ro = (int64_t)r * PUSH_THREADS;
        bulk_g2s(stpos + s * PUSH_THREADS, rgpos + ro, PUSH_THREADS * 16, &full_bar[s]);
        bulk_g2s(stvx + s * PUSH_THREADS, rgvx + ro, PUSH_THREADS * 4, &full_bar[s]);
        bulk_g2s(stvy + s * PUSH_THREADS, rgvy + ro, PUSH_THREADS * 4, &full_bar[s]);
        bulk_g2s(stvz + s * PUSH_THREADS, rgvz + ro, PUSH_THREADS * 4, &full_bar[s]);
        issued = r + 1;
      }
    }
    __syncwarp();
  } else {

  const float qmp = a.qmp[is], qfix = a.qfix[is];
  const float gustep = a.gustep, hr = 0.5f * a.rustep;
  // A particle can end inside a body without leaving its cell (entering a
  // cylinder or a sphere, or starting inside any body, where the reference's
  // end-point test absorbs it): in a tile region whose box touches a body's
  // cells (a box's lo..hi, its faces included; a curved body's bounding
  // cells), every particle takes the general path, whose absorption test is
  // the reference's (the in-cell test below then fails for all).
  float flo = 0.f;
  if (CURV)
    for (int q = 0; q < a.bd.n; q++) {
      bool hit = true;
#pragma unroll
      for (int d = 0; d < 3; d++) hit = hit && o[d] + B - 2 >= a.bd.lo[q][d] && o[d] <= a.bd.hi[q][d];
      if (hit) flo = 2.0f;
    }

  float acc[NC];
#pragma unroll
  for (int s = 0; s < NC; s++) acc[s] = 0.f;
  uint32_t runcell = DEAD;
  int runbase = -1;
  int nesc = 0;
  int rqn = 0, xqn = 0;  // warp-uniform queue lengths
  bool failed = false;
  int seen = 0;  // rows observed complete (thread 0)
  // Row r is pushed while row r+1 is already in shared memory: the cell of
  // the thread's next particle decides whether a change of cell starts a new
  // run or is a single particle out of place (one that changed cell since
  // the sort), which then takes the cross path and leaves the run intact.
  bool okme = false;
  if (L > 0) {
    okme = mbar_wait(&full_bar[0], 0u);
    if (!__any_sync(0xffffffffu, okme)) failed = true;
    for (int k = 0; !okme && k < 1024; k++) okme = mbar_try_wait(&full_bar[0], 0u);
    if (tid == 0 && okme) seen = 1;
  }

  int r = 0;
  for (;;) {
  // the stage of row r and the parity of its use, kept as running counters
  int s = r % NS;
  uint32_t ph = (uint32_t)((r / NS) & 1);
  for (; r < L && !failed; r++) {
    const int s1 = s + 1 == NS ? 0 : s + 1;
    const uint32_t par1 = s1 == 0 ? ph ^ 1u : ph;
    uint32_t nextcell = DEAD;
    bool oknext = false;
    if (r + 1 < L) {
      oknext = mbar_wait(&full_bar[s1], par1);
      if (!__any_sync(0xffffffffu, oknext)) {
        failed = true;
        break;
      }
      for (int k = 0; !oknext && k < 1024; k++) oknext = mbar_try_wait(&full_bar[s1], par1);
      if (tid == 0 && oknext) seen = r + 2;
      if (oknext) nextcell = (uint32_t)__float_as_int(stpos[s1 * PUSH_THREADS + tid].w);
    }
    const float4 ps = stpos[s * PUSH_THREADS + tid];
    float vx = stvx[s * PUSH_THREADS + tid];
    float vy = stvy[s * PUSH_THREADS + tid];
    float vz = stvz[s * PUSH_THREADS + tid];
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty_bar[s]);

    const uint32_t cell = (uint32_t)__float_as_int(ps.w);
    bool act = cell != DEAD && okme;
    okme = oknext;
    int ib = 0, jb = 0, kb = 0;
    if (act) {
      unpack(g, cell, ib, jb, kb);
      if (ib >= g.nx || jb >= g.ny || kb >= g.nz) {
        report_bad(a.status, a.diag, SITE_FX_PUSH, slot0 + (int64_t)r * PUSH_THREADS + tid, (long long)cell);
        act = false;
      }
    }
    // ---- a new cell ends the thread's run (its sums go to the run queue)
    // when the next particle is in that cell too, or when there is no run
    const bool newrun = DEP && act && cell != runcell && (runbase < 0 || nextcell == cell || nextcell == DEAD);
    if (DEP) {
      const bool evict = newrun && runbase >= 0;
      const unsigned mk = __ballot_sync(0xffffffffu, evict);
      if (mk) {
        if (evict) {
          float* en = rq + (rqn + __popc(mk & lt)) * QW;
#pragma unroll
          for (int q = 0; q < NC; q++) en[q] = acc[q];
          en[NC] = __int_as_float(runbase);
        }
        rqn += __popc(mk);
        if (rqn >= RQ_DRAIN) {
          drain_runs<NC>(box, slot_off, rq, rqn, qfix, lane);
          rqn = 0;
        }
      }
    }
    // a new run starts from zero: folded into this particle's accumulate
    // below, or (rarely: the particle itself leaves the run's cell) cleared
    const float keep = newrun ? 0.f : 1.f;
    if (newrun) {
      runcell = cell;
      runbase = box_base<B>(o, ib, jb, kb);
    }

    // ---- gather + Buneman-Boris (psolve1.F90:186-272)
    bool simple = false, oop = false, defer = false;
    int gb = -1;
    float sx = 0.f, syy = 0.f, szz = 0.f;
    if (act) {
      gb = cell == runcell ? runbase : box_base<B>(o, ib, jb, kb);
      // a part of a step whose eb arrives in z chunks: a cell outside the box
      // (a particle that crossed a periodic face or left the box since the
      // sort) whose node planes are not converted yet is left as it is for
      // k_fx_deferred
      defer = PARTS && gb < 0 && kb + 1 > a.zready;
      if (defer) {
        const int64_t m = slot0 + (int64_t)r * PUSH_THREADS + tid;
        atomicOr(a.defer + (m >> 5), 1u << (m & 31));
      } else {
        kick<B>(a, sf0, sf1, gb, ib, jb, kb, ps, qmp, vx, vy, vz);
        sx = ps.x + vx * gustep;
        syy = ps.y + vy * gustep;
        szz = ps.z + vz * gustep;
        // an end point exactly on a cell face takes the general path (it may
        // lie on a body face: inclusive bounds)
        const bool incell = sx > flo && sx < 1.0f && syy > 0.f && syy < 1.0f && szz > 0.f && szz < 1.0f;
        simple = incell && (!DEP || (cell == runcell && runbase >= 0));
        // a particle that stays in its cell but is out of place in the thread's
        // run (it changed cell since the sort): its 20 sums go to the run queue
        oop = DEP && incell && !simple && gb >= 0;
      }
    }
    const unsigned om = DEP ? __ballot_sync(0xffffffffu, oop) : 0u;
    float* oen = oop ? rq + (rqn + __popc(om & lt)) * QW : nullptr;
    if (DEP && (simple || oop)) {
      // both zigzag segments in the same cell: relay point at the midpoint,
      // equal segment fluxes h = (a-b)/2/ustep, mid-points m -+ (a-b)/4; the
      // sum of the two bilinear weight sets is written with S = a+b, D = a-b
      float cv[NC];
      if (JD) {
        const float Sx = sx + ps.x, Sy = syy + ps.y, Sz = szz + ps.z;
        const float Dx = sx - ps.x, Dy = syy - ps.y, Dz = szz - ps.z;
        const float hx = Dx * hr, hy = Dy * hr, hz = Dz * hr;
        float P;
        P = 0.5f * Sy * Sz + 0.125f * Dy * Dz;
        cv[3] = hx * P; cv[1] = hx * (Sy - P); cv[2] = hx * (Sz - P); cv[0] = hx * (2.0f - Sy - Sz + P);
        P = 0.5f * Sx * Sz + 0.125f * Dx * Dz;
        cv[7] = hy * P; cv[5] = hy * (Sx - P); cv[6] = hy * (Sz - P); cv[4] = hy * (2.0f - Sx - Sz + P);
        P = 0.5f * Sx * Sy + 0.125f * Dx * Dy;
        cv[11 % NC] = hz * P; cv[9 % NC] = hz * (Sx - P); cv[10 % NC] = hz * (Sy - P);
        cv[8 % NC] = hz * (2.0f - Sx - Sy + P);
      }
      // CIC charge at the new position (charge.F90:152-210)
      const float XY = sx * syy, XZ = sx * szz, YZ = syy * szz, Z2 = 1.0f - szz, XZ2 = sx * Z2, YZ2 = syy * Z2;
      const float r2 = XY * szz, r6 = XY * Z2;
      const float r3 = YZ - r2, r7 = YZ2 - r6;
      cv[RO + 2] = r2; cv[RO + 1] = XZ - r2; cv[RO + 3] = r3; cv[RO + 0] = szz - XZ - r3;
      cv[RO + 6] = r6; cv[RO + 5] = XZ2 - r6; cv[RO + 7] = r7; cv[RO + 4] = Z2 - XZ2 - r7;
      if (oop) {
#pragma unroll
        for (int q = 0; q < NC; q++) oen[q] = cv[q];
        oen[NC] = __int_as_float(gb);
      } else {
#pragma unroll
        for (int q = 0; q < NC; q++) acc[q] = fmaf(acc[q], keep, cv[q]);
      }
    }
    if (newrun && !simple) {
#pragma unroll
      for (int q = 0; q < NC; q++) acc[q] = 0.f;
    }
    // the new velocity of every particle (a cell-crossing one keeps its old
    // position until the general path writes the whole record)
    if (act && !defer) {
      const int m = r * PUSH_THREADS + tid;
      if (simple || oop) gpos[m] = make_float4(sx, syy, szz, ps.w);
      gvx[m] = vx;
      gvy[m] = vy;
      gvz[m] = vz;
    } else if (!DEP) {
      // a move-only step may write into other arrays than it reads: empty
      // and dead slots are carried over
      const int m = r * PUSH_THREADS + tid;
      gpos[m] = ps;
      gvx[m] = vx;
      gvy[m] = vy;
      gvz[m] = vz;
    }
    if (om) {
      rqn += __popc(om);
      if (rqn >= RQ_DRAIN) {
        drain_runs<NC>(box, slot_off, rq, rqn, qfix, lane);
        rqn = 0;
      }
    }
    // ---- cell-crossing particles: the warp's cross list (their positions
    // stay as they were; the general path after the row loop moves them)
    const bool cross = act && !simple && !oop && !defer;
    const unsigned xm = __ballot_sync(0xffffffffu, cross);
    if (xm) {
      if (cross) xl[xqn + __popc(xm & lt)] = r * PUSH_THREADS + tid;
      xqn += __popc(xm);
      if (xqn > XLCAP - 32) {  // full: empty it, then go on with the next row
        r++;
        break;
      }
    }
    s = s1;
    ph = par1;
  }
  if (xqn) {
    nesc += cross_list<B, DEP, CURV, JD>(a, is, slot0, box, o, xl, xqn, lane);
    xqn = 0;
  }
  if (r >= L || failed) break;
  }
  if (failed) report_bad(a.status, a.diag, SITE_FX_PUSH, -3, t);
  // the last run of every thread, and what is left in the queues
  if (DEP) {
    const bool has = runbase >= 0;
    const unsigned mk = __ballot_sync(0xffffffffu, has);
    if (has) {
      float* en = rq + (rqn + __popc(mk & lt)) * QW;
#pragma unroll
      for (int q = 0; q < NC; q++) en[q] = acc[q];
      en[NC] = __int_as_float(runbase);
    }
    rqn += __popc(mk);
    if (rqn) drain_runs<NC>(box, slot_off, rq, rqn, qfix, lane);
  }
  if (nesc) atomicAdd(&a.nesc[is], nesc);
  if (tid == 0) rows_seen = seen;
  }  // pushing warps
  __syncthreads();
  // copies still in flight after a failed wait complete before the CTA exits
  if (warp == PUSH_WARPS && lane == 0)
    for (int r = rows_seen; r < issued; r++) (void)mbar_wait(&full_bar[r % NS], (uint32_t)((r / NS) & 1));
  // add the tile accumulator into the global int64 arrays
  if (DEP) {
    for (int e = tid; e < NACC; e += PUSH_BLOCK) {
      unsigned long long v = box[e];
      if (v == 0ull) continue;
      int li = e % B, lj = (e / B) % B, lk = (e / (B * B)) % B, comp = e / (B * B * B);
      int i = o[0] + li, j = o[1] + lj, k = o[2] + lk;
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
}

// The row chunks of every tile region: cs[t] = first chunk of tile t,
// cs[ntiles] = the number of chunks (one block of 1024 threads per species).
__global__ void __launch_bounds__(1024) k_push_chunks(const int64_t* __restrict__ tile_start, int64_t ntiles,
                                                      int64_t* chunk_start, int chunk_rows) {
  __shared__ int64_t pa[1024];
  const int64_t* ts = tile_start + (int64_t)blockIdx.x * (ntiles + 1);
  int64_t* cs = chunk_start + (int64_t)blockIdx.x * (ntiles + 1);
  const int tid = threadIdx.x;
  const int64_t per = (ntiles + 1023) / 1024;
  const int64_t t0 = tid * per, t1 = min(ntiles, t0 + per);
  auto chunks = [&](int64_t t) {
    const int64_t rows = (ts[t + 1] - ts[t] + PUSH_THREADS - 1) / PUSH_THREADS;
    return (rows + chunk_rows - 1) / chunk_rows;
  };
  int64_t sa = 0;
  for (int64_t t = t0; t < t1; t++) sa += chunks(t);
  pa[tid] = sa;
  __syncthreads();
  for (int d = 1; d < 1024; d <<= 1) {
    const int64_t v = tid >= d ? pa[tid - d] : 0;
    __syncthreads();
    pa[tid] += v;
    __syncthreads();
  }
  int64_t ra = pa[tid] - sa;
  for (int64_t t = t0; t < t1; t++) {
    cs[t] = ra;
    ra += chunks(t);
  }
  if (tid == 1023) cs[ntiles] = pa[1023];
}

// Injected particles of the tail zone of species `is`, one thread each: the
// random fraction of the step for a particle injected since the last push
// (psolve1.F90:150-156: gustep = ustep * U), gather from the global node
// field, Buneman-Boris, and the general path with global deposits.
template <bool JD>
__global__ void k_fx_tail(FxPushArgs a, int is, int64_t tail0, int64_t ntail, int32_t* ord, int ustep,
                          const double* randoms, int64_t nrand, const int64_t* rand_pos, int64_t ord_base,
                          uint64_t seed, uint64_t stream, int* nesc_out) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ntail) return;
  const Geo& g = a.g;
  const int64_t base = a.off[is];
  const int64_t slot = tail0 + k;
  const float4 ps = a.pos[base + slot];
  const uint32_t cell = (uint32_t)__float_as_int(ps.w);
  if (cell == DEAD) return;
  int ib, jb, kb;
  unpack(g, cell, ib, jb, kb);
  if (ib >= g.nx || jb >= g.ny || kb >= g.nz) {
    report_bad(a.status, a.diag, SITE_FX_PUSH, base + slot, (long long)cell);
    return;
  }
  float gus = (float)ustep;
  const int32_t o1 = ord[k];
  if (o1 > 0) {
    double u;
    const int64_t j = ord_base + o1 - 1;
    if (randoms) {
      const int64_t r = *rand_pos + j;
      if (r >= nrand) {
        atomicOr(a.status, ST_RANDOMS);
        u = 0.0;
      } else {
        u = randoms[r];
      }
    } else {
      u = hash_u01(seed, stream, (uint64_t)j);
    }
    gus = (float)((double)ustep * u);
    ord[k] = 0;
  }
  const float qmp = (float)((double)a.qmp[is] / (double)a.gustep * (double)gus);
  float vx = a.vx[base + slot], vy = a.vy[base + slot], vz = a.vz[base + slot];
  const float x1 = ps.x, y1 = ps.y, z1 = ps.z;
  const float xy1 = x1 * y1, xz1 = x1 * z1, yz1 = y1 * z1, z2 = 1.0f - z1;
  const float xz2 = x1 * z2, yz2 = y1 * z2;
  float wv[8];
  wv[2] = xy1 * z1; wv[1] = xz1 - wv[2]; wv[3] = yz1 - wv[2]; wv[0] = z1 - xz1 - wv[3];
  wv[6] = xy1 * z2; wv[5] = xz2 - wv[6]; wv[7] = yz2 - wv[6]; wv[4] = z2 - xz2 - wv[7];
  float fe[3], fb[3];
  const int64_t sy = g.nx + 1, sz = (int64_t)(g.nx + 1) * (g.ny + 1);
  gather8<false>(a.f0, a.f1, ib + sy * jb + sz * kb, sy, sz, wv, fe, fb);
  const float eex = fe[0] * qmp, eey = fe[1] * qmp, eez = fe[2] * qmp;
  const float bbx = fb[0] * qmp, bby = fb[1] * qmp, bbz = fb[2] * qmp;
  const float boris = 2.0f / (1.0f + bbx * bbx + bby * bby + bbz * bbz);
  vx += eex; vy += eey; vz += eez;
  const float vxt = vx + vy * bbz - vz * bby;
  const float vyt = vy + vz * bbx - vx * bbz;
  const float vzt = vz + vx * bby - vy * bbx;
  vx += boris * (vyt * bbz - vzt * bby);
  vy += boris * (vzt * bbx - vxt * bbz);
  vz += boris * (vxt * bby - vyt * bbx);
  vx += eex; vy += eey; vz += eez;
  const Sink sk{a.acc_rho, a.acc_j, a.fr, a.fj, g.nx, g.ny, g.nz, a.status, a.diag};
  const CrossCtx c{a.pos + base, a.vx + base, a.vy + base, a.vz + base, gus, a.rustep, a.qfix[is],
                   {a.npbnd[is][0], a.npbnd[is][1], a.npbnd[is][2]}, &a.bd, a.gc,
                   a.surf + (int64_t)is * a.bd.nsurf, is, base, a.ob.rec ? &a.ob : nullptr, a.status};
  const float en[XQW] = {__int_as_float((int)slot), ps.w, ps.x, ps.y, ps.z, vx, vy, vz};
  const int far[3] = {-(1 << 28), -(1 << 28), -(1 << 28)};  // no box: global deposits
  const int esc = cross_one<11, true, true, JD>(g, nullptr, far, sk, c, en);
  if (esc) atomicAdd(nesc_out, esc);
}

// The particles the parts of a step left for later (FxPushArgs::defer: a
// gather from node planes converted after their part ran), once every plane
// is converted: what the row loop and the general path do for a particle
// whose cell lies outside its tile's box -- the global gather and the kick,
// then the general path with global deposits (a deposit takes the same
// int64 value per node as through a tile's box).  The compiler may round
// this kernel's kick otherwise than the row loop's (where it fuses a
// multiply with an add), so such a particle can differ in the last bit from
// the same step pushed in one launch.  One thread per 32-slot word of the
// bitmap, which it clears.
template <int T, bool CURV, bool JD>
__global__ void k_fx_deferred(FxPushArgs a, uint32_t* __restrict__ bits, int64_t nwords, int nspec) {
  constexpr int B = T + 2 * PG + 1;
  const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= nwords) return;
  uint32_t m = bits[w];
  if (m == 0u) return;
  bits[w] = 0u;
  const Geo& g = a.g;
  const Sink sk{a.acc_rho, a.acc_j, a.fr, a.fj, g.nx, g.ny, g.nz, a.status, a.diag};
  const int far[3] = {-(1 << 28), -(1 << 28), -(1 << 28)};  // no box: global deposits
  while (m) {
    const int64_t slot = w * 32 + (__ffs(m) - 1);
    m &= m - 1u;
    int is = 0;
    for (int s = 1; s < nspec; s++)
      if (slot >= a.off[s]) is = s;
    const int64_t base = a.off[is];
    const float4 ps = a.pos[slot];
    const uint32_t cell = (uint32_t)__float_as_int(ps.w);
    int ib, jb, kb;
    unpack(g, cell, ib, jb, kb);
    if (cell == DEAD || ib >= g.nx || jb >= g.ny || kb >= g.nz) {
      report_bad(a.status, a.diag, SITE_FX_PUSH, slot, (long long)cell);
      continue;
    }
    float vx = a.vx[slot], vy = a.vy[slot], vz = a.vz[slot];
    kick<B>(a, nullptr, nullptr, -1, ib, jb, kb, ps, a.qmp[is], vx, vy, vz);
    a.vx[slot] = vx;
    a.vy[slot] = vy;
    a.vz[slot] = vz;
    const CrossCtx c{a.pos + base, a.vx + base, a.vy + base, a.vz + base, a.gustep, a.rustep, a.qfix[is],
                     {a.npbnd[is][0], a.npbnd[is][1], a.npbnd[is][2]}, &a.bd, a.gc,
                     a.surf + (int64_t)is * a.bd.nsurf, is, base, a.ob.rec ? &a.ob : nullptr, a.status};
    const float en[XQW] = {__int_as_float((int)(slot - base)), ps.w, ps.x, ps.y, ps.z, vx, vy, vz};
    const int esc = cross_one<B, true, CURV, JD>(g, nullptr, far, sk, c, en);
    if (esc) atomicAdd(&a.nesc[is], esc);
  }
}

// The compiled box edge for the largest tile edge tmax (<= 8).
inline int fx_box_tile(int tmax) { return tmax <= 4 ? 4 : 8; }

// Dynamic shared memory of the push: int64 accumulator (4 components, or
// rho alone without the current), row ring, field tile, run queues and cross
// lists.
inline int fx_push_smem(int tmax, bool jd = true) {
  int B = fx_box_tile(tmax) + 2 * PG + 1;
  int nf = B * B * B;
  const int qw = (jd ? NJ + NR : NR) + 1;
  const int nbox = ((jd ? 4 : 1) * nf + 1) & ~1;  // as NBOX in k_fx_push
  return nbox * (int)sizeof(unsigned long long) + push_stages(jd) * (int)ROW_BYTES +
         nf * (int)(sizeof(float4) + sizeof(float2)) +
         PUSH_WARPS * (RQCAP * qw * (int)sizeof(float) + XLCAP * (int)sizeof(int));
}

// The pushing kernel (DEP = true) for a compiled box tile (4 or 8), runs
// with cylinders or spheres, and with (jd) or without the current.
using PushKernel = void (*)(FxPushArgs);
using DeferredKernel = void (*)(FxPushArgs, uint32_t*, int64_t, int);
inline DeferredKernel deferred_kernel(int box, bool curved, bool jd) {
  if (box == 4) {
    if (curved) return jd ? k_fx_deferred<4, true, true> : k_fx_deferred<4, true, false>;
    return jd ? k_fx_deferred<4, false, true> : k_fx_deferred<4, false, false>;
  }
  if (curved) return jd ? k_fx_deferred<8, true, true> : k_fx_deferred<8, true, false>;
  return jd ? k_fx_deferred<8, false, true> : k_fx_deferred<8, false, false>;
}

template <bool PARTS>
inline PushKernel push_kernel_t(int box, bool curved, bool jd) {
  if (box == 4) {
    if (curved) return jd ? k_fx_push<4, true, true, true, PARTS> : k_fx_push<4, true, true, false, PARTS>;
    return jd ? k_fx_push<4, true, false, true, PARTS> : k_fx_push<4, true, false, false, PARTS>;
  }
  if (curved) return jd ? k_fx_push<8, true, true, true, PARTS> : k_fx_push<8, true, true, false, PARTS>;
  return jd ? k_fx_push<8, true, false, true, PARTS> : k_fx_push<8, true, false, false, PARTS>;
}
inline PushKernel push_kernel(int box, bool curved, bool jd, bool parts = false) {
  return parts ? push_kernel_t<true>(box, curved, jd) : push_kernel_t<false>(box, curved, jd);
}
