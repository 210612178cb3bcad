// fx_push.cuh -- the fused push + zigzag current + CIC charge kernel of the
// FP32 / fixed-point form (included by fx.cu inside its private namespace).
//
// One CTA (512 threads) pushes the particles that the last sort placed in
// one cell tile of one species.  At the start it copies the tile's FP32 E/B
// nodes (tile + 1-node guard) into shared memory, so the 8-corner gathers
// read shared memory.  The tile's particles are split into 512 contiguous
// slices, one per thread; because they are sorted by cell, a thread meets
// long runs of particles in the same cell.  A thread keeps the 20 deposits of
// a cell (12 zigzag-current and 8 CIC-charge node values) in FP32 registers
// while the cell does not change.  When the
// cell changes (the thread's run moves on), or a particle changes cell
// during the step (its "after" half), the thread appends the 20 values
// and the cell to its warp's queue in shared memory; when the queue holds 16
// or more entries the warp empties it together, one entry per lane, adding
// the values into the CTA's int64 tile accumulator (tile + 1-cell guard).
// So the conversions and atomics run with all lanes busy instead of one
// lane at a time.  The CTA finally adds its accumulator into the global
// int64 arrays.  Particle records move through shared memory: slices are
// loaded and stored with coalesced accesses in chunks of RUN particles.
//
// The tile edge T is a template parameter, so every node offset inside the
// accumulator is an immediate.  Deposits or gathers whose cell lies outside
// the tile box (particles that drifted more than one cell since the sort)
// take a separate path through the global arrays.

constexpr int PUSH_THREADS = 512;
constexpr int PUSH_WARPS = PUSH_THREADS / 32;
constexpr int PG = 1;           // guard cells around the tile
constexpr int QCAP = 48;        // queue entries per warp
constexpr int QW = 21;          // words per entry: 20 values + cell
constexpr int RUN = 4;          // particles per thread per staged chunk
constexpr int SLOT = RUN + 1;   // padded slots per thread (conflict-free reads)
constexpr int NJ = 12;          // zigzag node values of one cell
constexpr int NR = 8;           // CIC node values of one cell

struct FxPushArgs {
  float4* pos;                  // all species regions
  float* vx;
  float* vy;
  float* vz;
  const int64_t* tile_start;    // [nspec][ntiles+1], offsets inside each region
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
  int* nesc;                    // counter nesc(is), one int per species
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

// Global arrays for deposits whose cell lies outside the tile box.
struct Sink {
  unsigned long long* acc_rho;
  unsigned long long* acc_j;
  FieldDesc fr, fj;
  int nx, ny, nz;
  int* status;
  long long* diag;
};
struct V12 { float v[NJ]; };
struct V8 { float v[NR]; };

// Out-of-box bundles: global int64 atomics with bounds checks (rare path;
// values come by value so the callers' register arrays keep no address).
__device__ __noinline__ void put_j_global(Sink s, int i, int j, int k, V12 v, float qfix) {
  for (int q = 0; q < NJ; q++) {
    int ii = i + jdi(q), jj = j + jdj(q), kk = k + jdk(q);
    if (ii < -4 || jj < -4 || kk < -4 || ii > s.nx + 4 || jj > s.ny + 4 || kk > s.nz + 4) {
      report_bad(s.status, s.diag, SITE_FX_DEPOSIT, -2, ii + 100000LL * jj + 10000000000LL * kk);
      continue;
    }
    atomicAdd(&s.acc_j[s.fj.at(jcomp(q) - 1, ii, jj, kk)], (unsigned long long)to_fix(v.v[q], qfix));
  }
}

__device__ __noinline__ void put_r_global(Sink s, int i, int j, int k, V8 v, float qfix) {
  for (int r = 0; r < NR; r++) {
    int ii = i + rdi(r), jj = j + rdj(r), kk = k + rdk(r);
    if (ii < -1 || jj < -1 || kk < -1 || ii > s.nx + 1 || jj > s.ny + 1 || kk > s.nz + 1) {
      report_bad(s.status, s.diag, SITE_FX_DEPOSIT, -1, ii + 100000LL * jj + 10000000000LL * kk);
      continue;
    }
    atomicAdd(&s.acc_rho[s.fr.at(0, ii, jj, kk)], (unsigned long long)to_fix(v.v[r], qfix));
  }
}

// Box index of cell (i,j,k) when its 2x2x2 node block lies inside the box,
// else -1.
template <int B>
__device__ __forceinline__ int box_base(const int (&o)[3], int i, int j, int k) {
  int li = i - o[0], lj = j - o[1], lk = k - o[2];
  bool ok = (unsigned)li < (unsigned)(B - 1) && (unsigned)lj < (unsigned)(B - 1) && (unsigned)lk < (unsigned)(B - 1);
  return ok ? (lk * B + lj) * B + li : -1;
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

// A queued bundle whose cell lies outside the tile box (rare).
__device__ __noinline__ void put_bundle_global(Sink sk, int i, int j, int k, const float* en, float qfix) {
  V12 wj;
  V8 wr;
  for (int s = 0; s < NJ; s++) wj.v[s] = en[s];
  for (int r = 0; r < NR; r++) wr.v[r] = en[NJ + r];
  put_j_global(sk, i, j, k, wj, qfix);
  put_r_global(sk, i, j, k, wr, qfix);
}

// Empties a warp queue: lane l takes entries l, l+32, ...  Each lane walks
// its entry's 20 slots starting at slot (lane mod 20), so lanes holding
// entries of the same cell add to different nodes at the same time.
template <int B>
__device__ __forceinline__ void drain_queue(const Sink& sk, const Geo& g, unsigned long long* box, const int (&o)[3],
                                            const int* slot_off, float* q, int qn, float qfix, int lane) {
  __syncwarp();
  const int rot = lane % (NJ + NR);
  for (int p = 0; p < qn; p += 32) {
    int e = p + lane;
    if (e < qn) {
      const float* en = q + e * QW;
      uint32_t key = (uint32_t)__float_as_int(en[NJ + NR]);
      int i, j, k;
      unpack(g, key, i, j, k);
      i -= 1; j -= 1; k -= 1;  // keys hold cells shifted by +1 (qkey)
      int base = box_base<B>(o, i, j, k);
      if (base >= 0) {
#pragma unroll 4
        for (int s = 0; s < NJ + NR; s++) {
          int slot = s + rot;
          slot -= slot >= NJ + NR ? NJ + NR : 0;
          long long v = to_fix(en[slot], qfix);
          if (v) atomicAdd(&box[base + slot_off[slot]], (unsigned long long)v);
        }
      } else {
        put_bundle_global(sk, i, j, k, en, qfix);
      }
    }
  }
  __syncwarp();
}

// Cell key of an "after" bundle: cells may be -1 or n on an axis (the
// reference's guard indices), so the queue stores the cell shifted by +1.
__device__ __forceinline__ uint32_t qkey(const Geo& g, int i, int j, int k) { return pack(g, i + 1, j + 1, k + 1); }

template <int T>
__global__ void __launch_bounds__(PUSH_THREADS, 1) k_fx_push(FxPushArgs a) {
  constexpr int B = T + 2 * PG + 1;  // box and field tile edge (nodes)
  constexpr int NBOX = 4 * B * B * B;
  constexpr int NF = B * B * B;
  extern __shared__ unsigned long long smem[];
  __shared__ int slot_off[NJ + NR];
  const Geo& g = a.g;
  const int is = blockIdx.y;
  const int t = blockIdx.x;
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const unsigned lt = (1u << lane) - 1u;
  int tx = t % g.nt[0], ty = (t / g.nt[0]) % g.nt[1], tz = t / (g.nt[0] * g.nt[1]);
  // T bounds every tile edge; the box may be larger than a thin tile needs
  const int o[3] = {tx * g.t[0] - PG, ty * g.t[1] - PG, tz * g.t[2] - PG};
  unsigned long long* box = smem;
  float4* sf0 = reinterpret_cast<float4*>(smem + NBOX);
  float4* spos = sf0 + NF;
  float2* sf1 = reinterpret_cast<float2*>(spos + PUSH_THREADS * SLOT);
  float* svx = reinterpret_cast<float*>(sf1 + NF);
  float* svy = svx + PUSH_THREADS * SLOT;
  float* svz = svy + PUSH_THREADS * SLOT;
  float* queue = svz + PUSH_THREADS * SLOT + warp * QCAP * QW;

  const int64_t* ts = a.tile_start + (int64_t)is * (a.ntiles + 1);
  const int64_t p0 = ts[t], n = ts[t + 1] - p0;
  if (n <= 0) return;
  const int64_t sy = g.nx + 1, sz = (int64_t)(g.nx + 1) * (g.ny + 1);
  if (tid < NJ + NR) slot_off[tid] = tid < NJ ? BoxT<B>::joff(tid) : BoxT<B>::roff(tid - NJ);
  for (int e = tid; e < NBOX; e += PUSH_THREADS) box[e] = 0ull;
  // field tile: nodes o .. o+B-1 (those inside 0..n)
  for (int e = tid; e < NF; e += PUSH_THREADS) {
    int li = e % B, lj = (e / B) % B, lk = e / (B * B);
    int gi = o[0] + li, gj = o[1] + lj, gk = o[2] + lk;
    float4 p = make_float4(0.f, 0.f, 0.f, 0.f), q = p;
    if (gi >= 0 && gj >= 0 && gk >= 0 && gi <= g.nx && gj <= g.ny && gk <= g.nz) {
      int64_t gn = gi + sy * gj + sz * gk;
      p = __ldg(&a.f0[gn]);
      q = __ldg(&a.f1[gn]);
    }
    sf0[e] = p;
    sf1[e] = make_float2(q.x, q.y);
  }

  const int64_t off = a.off[is];
  float4* gpos = a.pos + off;
  float* gvx = a.vx + off;
  float* gvy = a.vy + off;
  float* gvz = a.vz + off;
  const float qmp = a.qmp[is], qfix = a.qfix[is];
  const int nb0 = a.npbnd[is][0], nb1 = a.npbnd[is][1], nb2 = a.npbnd[is][2];
  const Sink sk{a.acc_rho, a.acc_j, a.fr, a.fj, g.nx, g.ny, g.nz, a.status, a.diag};
  // thread slices of the tile's particles
  const int64_t s0 = p0 + (n * tid) / PUSH_THREADS;
  const int64_t s1 = p0 + (n * (tid + 1)) / PUSH_THREADS;
  const int64_t maxlen = (n + PUSH_THREADS - 1) / PUSH_THREADS;
  const int chunks = (int)((maxlen + RUN - 1) / RUN);

  float acc[NJ + NR];
#pragma unroll
  for (int s = 0; s < NJ + NR; s++) acc[s] = 0.f;
  uint32_t acckey = DEAD;
  int nesc = 0;
  int qn = 0;  // warp-uniform queue length

  for (int c = 0; c < chunks; c++) {
    __syncthreads();  // staging free; box and field tile ready on the first pass
#pragma unroll
    for (int r = 0; r < RUN; r++) {
      int e = tid + r * PUSH_THREADS;
      int ow = e / RUN, j = e % RUN;
      int64_t so = p0 + (n * ow) / PUSH_THREADS, se = p0 + (n * (ow + 1)) / PUSH_THREADS;
      int64_t m = so + (int64_t)c * RUN + j;
      if (m < se) {
        spos[ow * SLOT + j] = gpos[m];
        svx[ow * SLOT + j] = gvx[m];
        svy[ow * SLOT + j] = gvy[m];
        svz[ow * SLOT + j] = gvz[m];
      }
    }
    __syncthreads();
#pragma unroll 1
    for (int j = 0; j < RUN; j++) {
      int64_t m = s0 + (int64_t)c * RUN + j;
      bool act = m < s1;
      float4 ps = act ? spos[tid * SLOT + j] : make_float4(0.f, 0.f, 0.f, 0.f);
      uint32_t cell = act ? (uint32_t)__float_as_int(ps.w) : DEAD;
      act = act && cell != DEAD;
      int ib = 0, jb = 0, kb = 0;
      if (act) {
        unpack(g, cell, ib, jb, kb);
        if (ib >= g.nx || jb >= g.ny || kb >= g.nz) {
          report_bad(a.status, a.diag, SITE_FX_PUSH, m, (long long)cell);
          act = false;
        }
      }
      // ---- the register run follows cell_b; a new cell sends the old sums
      // through the warp queue
      uint32_t key = qkey(g, ib, jb, kb);
      {
        bool evict = act && key != acckey && acckey != DEAD;
        unsigned mk = __ballot_sync(0xffffffffu, evict);
        if (mk) {
          if (evict) {
            float* en = queue + (qn + __popc(mk & lt)) * QW;
#pragma unroll
            for (int s = 0; s < NJ + NR; s++) en[s] = acc[s];
            en[NJ + NR] = __int_as_float((int)acckey);
          }
          qn += __popc(mk);
          if (qn >= 16) {
            drain_queue<B>(sk, g, box, o, slot_off, queue, qn, qfix, lane);
            qn = 0;
          }
        }
      }
      if (act && key != acckey) {
#pragma unroll
        for (int s = 0; s < NJ + NR; s++) acc[s] = 0.f;
        acckey = key;
      }

      // ---- push
      Axis ax{}, ay{}, az{};
      bool simple = true, dead = false;
      float xd2 = 0.f, yd2 = 0.f, zd2 = 0.f, vvx2 = 0.f, vvy2 = 0.f, vvz2 = 0.f;
      if (act) {
        float vx = svx[tid * SLOT + j], vy = svy[tid * SLOT + j], vz = svz[tid * SLOT + j];
        // trilinear weights (psolve1.F90:186-199)
        float x1 = ps.x, y1 = ps.y, z1 = ps.z;
        float xy1 = x1 * y1, xz1 = x1 * z1, yz1 = y1 * z1, z2 = 1.0f - z1;
        float xz2 = x1 * z2, yz2 = y1 * z2;
        float wv[8];
        wv[2] = xy1 * z1; wv[1] = xz1 - wv[2]; wv[3] = yz1 - wv[2]; wv[0] = z1 - xz1 - wv[3];
        wv[6] = xy1 * z2; wv[5] = xz2 - wv[6]; wv[7] = yz2 - wv[6]; wv[4] = z2 - xz2 - wv[7];
        float eb_e[3], eb_b[3];
        int li = ib - o[0], lj = jb - o[1], lk = kb - o[2];
        if ((unsigned)li < (unsigned)(B - 1) && (unsigned)lj < (unsigned)(B - 1) && (unsigned)lk < (unsigned)(B - 1))
          gather8<true>(sf0, sf1, li + B * lj + (int64_t)B * B * lk, B, (int64_t)B * B, wv, eb_e, eb_b);
        else
          gather8<false>(a.f0, a.f1, ib + sy * jb + sz * kb, sy, sz, wv, eb_e, eb_b);
        // Buneman-Boris (psolve1.F90:247-272)
        float eex = eb_e[0] * qmp, eey = eb_e[1] * qmp, eez = eb_e[2] * qmp;
        float bbx = eb_b[0] * qmp, bby = eb_b[1] * qmp, bbz = eb_b[2] * qmp;
        float boris = 2.0f / (1.0f + bbx * bbx + bby * bby + bbz * bbz);
        vx += eex; vy += eey; vz += eez;
        float vxt = vx + vy * bbz - vz * bby;
        float vyt = vy + vz * bbx - vx * bbz;
        float vzt = vz + vx * bby - vy * bbx;
        vx += boris * (vyt * bbz - vzt * bby);
        vy += boris * (vzt * bbx - vxt * bbz);
        vz += boris * (vxt * bby - vyt * bbx);
        vx += eex; vy += eey; vz += eez;
        ax = axis_move(ib, ps.x, vx * a.gustep, g.nx, nb0);
        ay = axis_move(jb, ps.y, vy * a.gustep, g.ny, nb1);
        az = axis_move(kb, ps.z, vz * a.gustep, g.nz, nb2);
        if (ax.flip) vx = -vx;
        if (ay.flip) vy = -vy;
        if (az.flip) vz = -vz;
        dead = ax.dead || ay.dead || az.dead;
        if (dead) nesc++;
        uint32_t nc = dead ? DEAD : pack(g, ax.nc, ay.nc, az.nc);
        spos[tid * SLOT + j] = make_float4(ax.nf, ay.nf, az.nf, __int_as_float((int)nc));
        svx[tid * SLOT + j] = vx;
        svy[tid * SLOT + j] = vy;
        svz[tid * SLOT + j] = vz;
        // zigzag (psolve1.F90:717-757), integer parts first; segment 1 goes
        // to the run of cell_b
        float xd1 = ((float)(ax.rc - ib) + ax.rf + ps.x) * 0.5f;
        float yd1 = ((float)(ay.rc - jb) + ay.rf + ps.y) * 0.5f;
        float zd1 = ((float)(az.rc - kb) + az.rf + ps.z) * 0.5f;
        float vvx1 = ((float)(ax.rc - ib) + (ax.rf - ps.x)) * a.rustep;
        float vvy1 = ((float)(ay.rc - jb) + (ay.rf - ps.y)) * a.rustep;
        float vvz1 = ((float)(az.rc - kb) + (az.rf - ps.z)) * a.rustep;
        float w;
        w = yd1 * zd1; acc[3] += vvx1 * w; acc[1] += vvx1 * (yd1 - w); acc[2] += vvx1 * (zd1 - w); acc[0] += vvx1 * (1.0f - yd1 - (zd1 - w));
        w = xd1 * zd1; acc[7] += vvy1 * w; acc[5] += vvy1 * (xd1 - w); acc[6] += vvy1 * (zd1 - w); acc[4] += vvy1 * (1.0f - xd1 - (zd1 - w));
        w = xd1 * yd1; acc[11] += vvz1 * w; acc[9] += vvz1 * (xd1 - w); acc[10] += vvz1 * (yd1 - w); acc[8] += vvz1 * (1.0f - xd1 - (yd1 - w));
        xd2 = ((float)(ax.ac - ax.ia) + ax.af + (float)(ax.rc - ax.ia) + ax.rf) * 0.5f;
        yd2 = ((float)(ay.ac - ay.ia) + ay.af + (float)(ay.rc - ay.ia) + ay.rf) * 0.5f;
        zd2 = ((float)(az.ac - az.ia) + az.af + (float)(az.rc - az.ia) + az.rf) * 0.5f;
        vvx2 = ((float)(ax.ac - ax.rc) + (ax.af - ax.rf)) * a.rustep;
        vvy2 = ((float)(ay.ac - ay.rc) + (ay.af - ay.rf)) * a.rustep;
        vvz2 = ((float)(az.ac - az.rc) + (az.af - az.rf)) * a.rustep;
        simple = !ax.crossed && !ay.crossed && !az.crossed && ax.ia == ib && ay.ia == jb && az.ia == kb;
      }
      // ---- segment 2 and the charge: into the run when the cell did not
      // change, else through the warp queue
      bool cross = act && !simple;
      unsigned mk = __ballot_sync(0xffffffffu, cross);
      float* en = cross ? queue + (qn + __popc(mk & lt)) * QW : nullptr;
      if (act) {
        float J2[NJ], R[NR];
        float w;
        w = yd2 * zd2; J2[3] = vvx2 * w; J2[1] = vvx2 * (yd2 - w); J2[2] = vvx2 * (zd2 - w); J2[0] = vvx2 * (1.0f - yd2 - (zd2 - w));
        w = xd2 * zd2; J2[7] = vvy2 * w; J2[5] = vvy2 * (xd2 - w); J2[6] = vvy2 * (zd2 - w); J2[4] = vvy2 * (1.0f - xd2 - (zd2 - w));
        w = xd2 * yd2; J2[11] = vvz2 * w; J2[9] = vvz2 * (xd2 - w); J2[10] = vvz2 * (yd2 - w); J2[8] = vvz2 * (1.0f - xd2 - (yd2 - w));
        float X = ax.nf, Y = ay.nf, Z = az.nf;
        float XY = X * Y, XZ = X * Z, YZ = Y * Z, Z2 = 1.0f - Z, XZ2 = X * Z2, YZ2 = Y * Z2;
        R[2] = XY * Z; R[1] = XZ - R[2]; R[3] = YZ - R[2]; R[0] = Z - XZ - R[3];
        R[6] = XY * Z2; R[5] = XZ2 - R[6]; R[7] = YZ2 - R[6]; R[4] = Z2 - XZ2 - R[7];
        if (simple) {
#pragma unroll
          for (int s = 0; s < NJ; s++) acc[s] += J2[s];
#pragma unroll
          for (int r = 0; r < NR; r++) acc[NJ + r] += R[r];
        } else {
          // the stored cell differs from the after cell only at an outer
          // boundary (wrap or reflection): that charge goes out directly
          bool rsplit = dead || ax.nc != ax.ia || ay.nc != ay.ia || az.nc != az.ia;
          if (rsplit && !dead) {
            V8 wr;
#pragma unroll
            for (int r = 0; r < NR; r++) wr.v[r] = R[r];
            put_r_global(sk, ax.nc, ay.nc, az.nc, wr, qfix);
          }
#pragma unroll
          for (int s = 0; s < NJ; s++) en[s] = J2[s];
#pragma unroll
          for (int r = 0; r < NR; r++) en[NJ + r] = rsplit ? 0.f : R[r];
          en[NJ + NR] = __int_as_float((int)qkey(g, ax.ia, ay.ia, az.ia));
        }
      }
      if (mk) {
        qn += __popc(mk);
        if (qn >= 16) {
          drain_queue<B>(sk, g, box, o, slot_off, queue, qn, qfix, lane);
          qn = 0;
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RUN; r++) {
      int e = tid + r * PUSH_THREADS;
      int ow = e / RUN, j = e % RUN;
      int64_t so = p0 + (n * ow) / PUSH_THREADS, se = p0 + (n * (ow + 1)) / PUSH_THREADS;
      int64_t m = so + (int64_t)c * RUN + j;
      if (m < se) {
        gpos[m] = spos[ow * SLOT + j];
        gvx[m] = svx[ow * SLOT + j];
        gvy[m] = svy[ow * SLOT + j];
        gvz[m] = svz[ow * SLOT + j];
      }
    }
  }
  // the last run of every thread
  {
    bool has = acckey != DEAD;
    unsigned mk = __ballot_sync(0xffffffffu, has);
    if (has) {
      float* en = queue + (qn + __popc(mk & lt)) * QW;
#pragma unroll
      for (int s = 0; s < NJ + NR; s++) en[s] = acc[s];
      en[NJ + NR] = __int_as_float((int)acckey);
    }
    qn += __popc(mk);
    if (qn) drain_queue<B>(sk, g, box, o, slot_off, queue, qn, qfix, lane);
  }
  if (nesc) atomicAdd(&a.nesc[is], nesc);
  __syncthreads();
  // add the tile accumulator into the global int64 arrays
  for (int e = tid; e < NBOX; e += PUSH_THREADS) {
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

// The compiled box edge for the largest tile edge tmax (<= 8).
inline int fx_box_tile(int tmax) { return tmax <= 4 ? 4 : 8; }

inline int fx_push_smem(int tmax) {
  int B = fx_box_tile(tmax) + 2 * PG + 1;
  int nf = B * B * B;
  return 4 * nf * (int)sizeof(unsigned long long) + nf * (int)(sizeof(float4) + sizeof(float2)) +
         PUSH_THREADS * SLOT * (int)(sizeof(float4) + 3 * sizeof(float)) + PUSH_WARPS * QCAP * QW * (int)sizeof(float);
}
