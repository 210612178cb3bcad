// fx_push.cuh -- the fused push + zigzag current + CIC charge kernel of the
// FP32 / fixed-point form (included by fx.cu inside its private namespace).
//
// One CTA pushes the particles that the last sort placed in one cell tile of
// one species.  The tile's particles are split into 256 contiguous slices,
// one per thread; because they are sorted by cell, a thread meets long runs
// of particles in the same cell.  A thread keeps the 20 deposits of a cell
// (12 zigzag-current and 8 CIC-charge node values) in FP32 registers while
// the cell does not change, for up to two cells at a time (the least
// recently used one is written out first), and writes a cell's sums into the
// CTA's int64 tile accumulator (tile + 2-cell guard, shared memory) only when
// the cell leaves the pair.  Particles that change cell in this step add
// their "before" half (zigzag segment 1) to the run and write the rest
// directly.  The CTA finally adds its accumulator into the global int64
// arrays.  Particle records move through shared memory: slices are loaded
// and stored with coalesced accesses in chunks of RUN particles per thread.
//
// The tile edge T is a template parameter, so every node offset inside the
// accumulator is an immediate: a deposit is one FP32->int64 conversion and
// one shared-memory atomic.  Deposits whose cell lies outside the tile box
// (rare: particles that drifted more than the guard) take a separate,
// non-inlined path into the global arrays.

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

// 12 zigzag values starting at v[first] (compile-time indices only).
template <int B, int N>
__device__ __forceinline__ void put_j(const Sink& sk, unsigned long long* box, const int (&o)[3], int i, int j, int k,
                                      const float (&v)[N], int first_unused, float qfix) {
  int base = box_base<B>(o, i, j, k);
  if (base >= 0) {
#pragma unroll
    for (int q = 0; q < NJ; q++)
      atomicAdd(&box[base + BoxT<B>::joff(q)], (unsigned long long)to_fix(v[q], qfix));
  } else {
    V12 w;
#pragma unroll
    for (int q = 0; q < NJ; q++) w.v[q] = v[q];
    put_j_global(sk, i, j, k, w, qfix);
  }
}

// 8 charge values at v[OFF .. OFF+7].
template <int B, int OFF, int N>
__device__ __forceinline__ void put_r(const Sink& sk, unsigned long long* box, const int (&o)[3], int i, int j, int k,
                                      const float (&v)[N], float qfix) {
  int base = box_base<B>(o, i, j, k);
  if (base >= 0) {
#pragma unroll
    for (int r = 0; r < NR; r++)
      atomicAdd(&box[base + BoxT<B>::roff(r)], (unsigned long long)to_fix(v[OFF + r], qfix));
  } else {
    V8 w;
#pragma unroll
    for (int r = 0; r < NR; r++) w.v[r] = v[OFF + r];
    put_r_global(sk, i, j, k, w, qfix);
  }
}

// Writes the 20 register sums of one cell (key) and clears them.
template <int B>
__device__ __forceinline__ void flush_cell(const Sink& sk, const Geo& g, unsigned long long* box, const int (&o)[3],
                                           uint32_t key, float (&acc)[NJ + NR], float qfix) {
  if (key == DEAD) return;
  int i, j, k;
  unpack(g, key, i, j, k);
  put_j<B, NJ + NR>(sk, box, o, i, j, k, acc, 0, qfix);
  put_r<B, NJ, NJ + NR>(sk, box, o, i, j, k, acc, qfix);
#pragma unroll
  for (int q = 0; q < NJ + NR; q++) acc[q] = 0.f;
}

template <int T>
__global__ void __launch_bounds__(FX_THREADS, 2) k_fx_push(FxPushArgs a) {
  constexpr int B = T + 2 * GUARD + 1;
  constexpr int NBOX = 4 * B * B * B;
  extern __shared__ unsigned long long smem[];
  const Geo& g = a.g;
  const int is = blockIdx.y;
  const int t = blockIdx.x;
  const int tid = threadIdx.x;
  int tx = t % g.nt[0], ty = (t / g.nt[0]) % g.nt[1], tz = t / (g.nt[0] * g.nt[1]);
  // T bounds every tile edge; the box may be larger than a thin tile needs
  const int o[3] = {tx * g.t[0] - GUARD, ty * g.t[1] - GUARD, tz * g.t[2] - GUARD};
  unsigned long long* box = smem;
  float4* spos = reinterpret_cast<float4*>(smem + NBOX);
  float* svx = reinterpret_cast<float*>(spos + FX_THREADS * SLOT);
  float* svy = svx + FX_THREADS * SLOT;
  float* svz = svy + FX_THREADS * SLOT;

  const int64_t* ts = a.tile_start + (int64_t)is * (a.ntiles + 1);
  const int64_t p0 = ts[t], n = ts[t + 1] - p0;
  if (n <= 0) return;
  for (int e = tid; e < NBOX; e += FX_THREADS) box[e] = 0ull;

  const int64_t off = a.off[is];
  float4* gpos = a.pos + off;
  float* gvx = a.vx + off;
  float* gvy = a.vy + off;
  float* gvz = a.vz + off;
  const float qmp = a.qmp[is], qfix = a.qfix[is];
  const int nb0 = a.npbnd[is][0], nb1 = a.npbnd[is][1], nb2 = a.npbnd[is][2];
  // thread slices of the tile's particles
  const int64_t s0 = p0 + ((n * tid) >> 8);
  const int64_t s1 = p0 + ((n * (tid + 1)) >> 8);
  const int64_t maxlen = (n + FX_THREADS - 1) >> 8;
  const int chunks = (int)((maxlen + RUN - 1) / RUN);

  const Sink sk{a.acc_rho, a.acc_j, a.fr, a.fj, g.nx, g.ny, g.nz, a.status, a.diag};
  float accA[NJ + NR], accB[NJ + NR];
#pragma unroll
  for (int s = 0; s < NJ + NR; s++) { accA[s] = 0.f; accB[s] = 0.f; }
  uint32_t keyA = DEAD, keyB = DEAD;
  bool lastA = true;
  int nesc = 0;
  const int64_t sy = g.nx + 1, sz = (int64_t)(g.nx + 1) * (g.ny + 1);

  for (int c = 0; c < chunks; c++) {
    __syncthreads();  // staging buffers free (and box zeroed, on the first pass)
#pragma unroll
    for (int r = 0; r < RUN; r++) {
      int e = tid + r * FX_THREADS;
      int ow = e / RUN, j = e % RUN;
      int64_t so = p0 + ((n * ow) >> 8), se = p0 + ((n * (ow + 1)) >> 8);
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
      if (m >= s1) break;
      float4 ps = spos[tid * SLOT + j];
      uint32_t cell = (uint32_t)__float_as_int(ps.w);
      if (cell == DEAD) continue;
      int ib, jb, kb;
      unpack(g, cell, ib, jb, kb);
      if (ib >= g.nx || jb >= g.ny || kb >= g.nz) {
        report_bad(a.status, a.diag, SITE_FX_PUSH, m, (long long)cell);
        continue;
      }
      float vx = svx[tid * SLOT + j], vy = svy[tid * SLOT + j], vz = svz[tid * SLOT + j];
      // trilinear weights (psolve1.F90:186-199)
      float x1 = ps.x, y1 = ps.y, z1 = ps.z;
      float xy1 = x1 * y1, xz1 = x1 * z1, yz1 = y1 * z1, z2 = 1.0f - z1;
      float xz2 = x1 * z2, yz2 = y1 * z2;
      float v3 = xy1 * z1, v2 = xz1 - v3, v4 = yz1 - v3, v1 = z1 - xz1 - v4;
      float v7 = xy1 * z2, v6 = xz2 - v7, v8 = yz2 - v7, v5 = z2 - xz2 - v8;
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
      eex *= qmp; eey *= qmp; eez *= qmp;
      bbx *= qmp; bby *= qmp; bbz *= qmp;
      float boris = 2.0f / (1.0f + bbx * bbx + bby * bby + bbz * bbz);
      vx += eex; vy += eey; vz += eez;
      float vxt = vx + vy * bbz - vz * bby;
      float vyt = vy + vz * bbx - vx * bbz;
      float vzt = vz + vx * bby - vy * bbx;
      vx += boris * (vyt * bbz - vzt * bby);
      vy += boris * (vzt * bbx - vxt * bbz);
      vz += boris * (vxt * bby - vyt * bbx);
      vx += eex; vy += eey; vz += eez;
      Axis ax = axis_move(ib, ps.x, vx * a.gustep, g.nx, nb0);
      Axis ay = axis_move(jb, ps.y, vy * a.gustep, g.ny, nb1);
      Axis az = axis_move(kb, ps.z, vz * a.gustep, g.nz, nb2);
      if (ax.flip) vx = -vx;
      if (ay.flip) vy = -vy;
      if (az.flip) vz = -vz;
      bool dead = ax.dead || ay.dead || az.dead;
      // zigzag (psolve1.F90:717-757), integer parts first
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
      float J1[NJ], J2[NJ], R[NR];
      float w;
      w = yd1 * zd1; J1[3] = vvx1 * w; J1[1] = vvx1 * (yd1 - w); J1[2] = vvx1 * (zd1 - w); J1[0] = vvx1 * (1.0f - yd1 - (zd1 - w));
      w = xd1 * zd1; J1[7] = vvy1 * w; J1[5] = vvy1 * (xd1 - w); J1[6] = vvy1 * (zd1 - w); J1[4] = vvy1 * (1.0f - xd1 - (zd1 - w));
      w = xd1 * yd1; J1[11] = vvz1 * w; J1[9] = vvz1 * (xd1 - w); J1[10] = vvz1 * (yd1 - w); J1[8] = vvz1 * (1.0f - xd1 - (yd1 - w));
      w = yd2 * zd2; J2[3] = vvx2 * w; J2[1] = vvx2 * (yd2 - w); J2[2] = vvx2 * (zd2 - w); J2[0] = vvx2 * (1.0f - yd2 - (zd2 - w));
      w = xd2 * zd2; J2[7] = vvy2 * w; J2[5] = vvy2 * (xd2 - w); J2[6] = vvy2 * (zd2 - w); J2[4] = vvy2 * (1.0f - xd2 - (zd2 - w));
      w = xd2 * yd2; J2[11] = vvz2 * w; J2[9] = vvz2 * (xd2 - w); J2[10] = vvz2 * (yd2 - w); J2[8] = vvz2 * (1.0f - xd2 - (yd2 - w));
      {
        float X = ax.nf, Y = ay.nf, Z = az.nf;
        float XY = X * Y, XZ = X * Z, YZ = Y * Z, Z2 = 1.0f - Z, XZ2 = X * Z2, YZ2 = Y * Z2;
        R[2] = XY * Z; R[1] = XZ - R[2]; R[3] = YZ - R[2]; R[0] = Z - XZ - R[3];
        R[6] = XY * Z2; R[5] = XZ2 - R[6]; R[7] = YZ2 - R[6]; R[4] = Z2 - XZ2 - R[7];
      }
      if (dead) nesc++;
      uint32_t nc = dead ? DEAD : pack(g, ax.nc, ay.nc, az.nc);
      spos[tid * SLOT + j] = make_float4(ax.nf, ay.nf, az.nf, __int_as_float((int)nc));
      svx[tid * SLOT + j] = vx;
      svy[tid * SLOT + j] = vy;
      svz[tid * SLOT + j] = vz;

      // ---- deposit: segment 1 (and, without a cell change, everything)
      // goes to the register run of cell_b
      bool simple = !ax.crossed && !ay.crossed && !az.crossed && ax.ia == ib && ay.ia == jb && az.ia == kb;
      bool useA;
      if (cell == keyA) useA = true;
      else if (cell == keyB) useA = false;
      else if (lastA) {  // evict B
        flush_cell<B>(sk, g, box, o, keyB, accB, qfix);
        keyB = cell;
        useA = false;
      } else {
        flush_cell<B>(sk, g, box, o, keyA, accA, qfix);
        keyA = cell;
        useA = true;
      }
      lastA = useA;
      float sm = simple ? 1.0f : 0.0f;
#pragma unroll
      for (int s = 0; s < NJ; s++) {
        float v = fmaf(sm, J2[s], J1[s]);
        if (useA) accA[s] += v; else accB[s] += v;
      }
#pragma unroll
      for (int r = 0; r < NR; r++) {
        float v = sm * R[r];
        if (useA) accA[NJ + r] += v; else accB[NJ + r] += v;
      }
      if (!simple) {
        // segment 2 at the after cell, charge at the stored position
        put_j<B, NJ>(sk, box, o, ax.ia, ay.ia, az.ia, J2, 0, qfix);
        if (!dead) put_r<B, 0, NR>(sk, box, o, ax.nc, ay.nc, az.nc, R, qfix);
      }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RUN; r++) {
      int e = tid + r * FX_THREADS;
      int ow = e / RUN, j = e % RUN;
      int64_t so = p0 + ((n * ow) >> 8), se = p0 + ((n * (ow + 1)) >> 8);
      int64_t m = so + (int64_t)c * RUN + j;
      if (m < se) {
        gpos[m] = spos[ow * SLOT + j];
        gvx[m] = svx[ow * SLOT + j];
        gvy[m] = svy[ow * SLOT + j];
        gvz[m] = svz[ow * SLOT + j];
      }
    }
  }
  flush_cell<B>(sk, g, box, o, keyA, accA, qfix);
  flush_cell<B>(sk, g, box, o, keyB, accB, qfix);
  if (nesc) atomicAdd(&a.nesc[is], nesc);
  __syncthreads();
  // add the tile accumulator into the global int64 arrays
  for (int e = tid; e < NBOX; e += FX_THREADS) {
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
  int B = fx_box_tile(tmax) + 2 * GUARD + 1;
  return 4 * B * B * B * (int)sizeof(unsigned long long) + FX_THREADS * SLOT * (int)(sizeof(float4) + 3 * sizeof(float));
}

inline const void* fx_push_kernel(int tmax) {
  return fx_box_tile(tmax) == 4 ? (const void*)k_fx_push<4> : (const void*)k_fx_push<8>;
}
