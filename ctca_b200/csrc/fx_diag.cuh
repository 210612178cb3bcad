// fx_diag.cuh -- the FP64 checks of the FP32 / fixed-point form and the
// absorbed (background) charge (included by fx.cu inside its private
// namespace, after fx_push.cuh).
//
// * Kinetic energy (energy.F90:29-47): FP64 sums of vx^2, vy^2, vz^2 over
//   the live particles of a species region.  A v of FP32 squared is exact in
//   FP64; the sums run in a fixed order (per-block partials of a fixed grid,
//   then one block over the partials), so the result is reproducible bit for
//   bit.
// * Charge continuity (rhoupd.F90:41-49): when a step converts its folded
//   int64 rho into the FP64 rho field, the field still holds the rho of the
//   step before; k_fix_to_rho takes, over the nodes 0..n of every axis, the
//   FP64 residual |rho_new - rho_old + 2 (div J)| of the step (J already
//   converted) and keeps its largest value and that of |rho_new|.
// * Background charge (charge.F90:414-449 with rhobk(...,3) += rhobk(...,1)
//   of emses.F90:249-251): the exact int64 counts per surface cell of the
//   box bodies (absorbed minus emitted particles since the start) become the
//   node field rhobk: a surface cell's charge q * count goes in equal
//   quarters to the four nodes of its face cell.  The counts of the faces
//   that meet at a node are summed in int64 per species, then scaled once in
//   FP64, so the field is exact up to that one rounding.

constexpr int DIAG_BLOCK = 256;
constexpr int DIAG_GRID = 4 * 148;

// Per-block FP64 sums of v^2 per component over slots [0, ntile) of the
// tile regions (ntile read on the device: the last tile_pad entry) and the
// tail zone [tail0, tail0 + ntail) of one species region; dead and empty
// slots hold the DEAD cell.  part[blockIdx.x][3].
__global__ void __launch_bounds__(DIAG_BLOCK) k_fx_energy_part(const float4* __restrict__ pos,
                                                               const float* __restrict__ vx,
                                                               const float* __restrict__ vy,
                                                               const float* __restrict__ vz,
                                                               const int64_t* __restrict__ tile_end, int64_t tail0,
                                                               int64_t ntail, double* __restrict__ part) {
  __shared__ double s[3][DIAG_BLOCK / 32];
  const int64_t ntile = *tile_end;
  const int64_t n = ntile + ntail;
  double t[3] = {0.0, 0.0, 0.0};
  for (int64_t m = (int64_t)blockIdx.x * DIAG_BLOCK + threadIdx.x; m < n; m += (int64_t)gridDim.x * DIAG_BLOCK) {
    const int64_t slot = m < ntile ? m : tail0 + (m - ntile);
    if ((uint32_t)__float_as_int(pos[slot].w) == DEAD) continue;
    const double a = vx[slot], b = vy[slot], c = vz[slot];
    t[0] += a * a;
    t[1] += b * b;
    t[2] += c * c;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    double v = t[d];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) s[d][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double v = 0.0;
    for (int w = 0; w < DIAG_BLOCK / 32; w++) v += s[threadIdx.x][w];
    part[blockIdx.x * 3 + threadIdx.x] = v;
  }
}

// out[3] = the sums of the nparts partials, in order.
__global__ void k_fx_energy_sum(const double* __restrict__ part, int nparts, double* __restrict__ out) {
  if (threadIdx.x < 3) {
    double v = 0.0;
    for (int b = 0; b < nparts; b++) v += part[b * 3 + threadIdx.x];
    out[threadIdx.x] = v;
  }
}

// Largest of non-negative doubles, as their bit patterns (which order them).
__device__ __forceinline__ void max_nonneg(unsigned long long* p, double v) {
  atomicMax(p, (unsigned long long)__double_as_longlong(v));
}

// rho (FP64) from the folded int64 accumulator (scale 2^-40), and over the
// nodes 0..n the continuity residual of the step: res[0] = max |rho_new -
// rho_old + 2 (div J)|, res[1] = max |rho_new| (rhoupd.F90:41-49 gives
// rho_old - 2 div J as the prediction of rho_new).  The maxima are taken per
// block (warp shuffles, then the block's warps) before one atomic per block.
constexpr int RHO_BLOCK = 256;
__global__ void __launch_bounds__(RHO_BLOCK) k_fix_to_rho(const long long* __restrict__ acc, double* __restrict__ rho,
                                                          const double* __restrict__ aj, FieldDesc fr, FieldDesc fj,
                                                          int nx, int ny, int nz, unsigned long long* res) {
  __shared__ double wmax[2][RHO_BLOCK / 32];
  const int64_t e = (int64_t)blockIdx.x * RHO_BLOCK + threadIdx.x;
  double r = 0.0, m = 0.0;
  if (e < fr.size()) {
    const double v = (double)acc[e] * (1.0 / 1099511627776.0);
    const int64_t ex = fr.ex, ey = fr.ey;
    const int i = (int)(e % ex) + fr.lo, j = (int)((e / ex) % ey) + fr.lo, k = (int)(e / (ex * ey)) + fr.lo;
    if (i >= 0 && j >= 0 && k >= 0 && i <= nx && j <= ny && k <= nz) {
      if (aj) {  // without the step's current (the electrostatic step) no residual
        const double div = (aj[fj.at(0, i, j, k)] - aj[fj.at(0, i - 1, j, k)]) +
                           (aj[fj.at(1, i, j, k)] - aj[fj.at(1, i, j - 1, k)]) +
                           (aj[fj.at(2, i, j, k)] - aj[fj.at(2, i, j, k - 1)]);
        r = fabs(v - (rho[e] - div * 2.0));
      }
      m = fabs(v);
    }
    rho[e] = v;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    r = fmax(r, __shfl_down_sync(0xffffffffu, r, o));
    m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    wmax[0][warp] = r;
    wmax[1][warp] = m;
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    double v = 0.0;
    for (int w = 0; w < RHO_BLOCK / 32; w++) v = fmax(v, wmax[threadIdx.x][w]);
    if (v > 0.0) max_nonneg(&res[threadIdx.x], v);
  }
}

// One body's background charge: for every node of its bounding box (one
// thread each) the counts of the surface cells of species `is` whose face
// cell has the node as a corner, summed in int64, then rhobk(node) +=
// q * 0.25 * sum.  Faces as in Bodies: -x,+x,-y,+y,-z,+z, first tangential
// axis fastest.
__global__ void k_fx_background(const unsigned long long* __restrict__ surf, Bodies bd, int q, double qs,
                                double* __restrict__ rhobk, FieldDesc fr) {
  const int lo0 = bd.lo[q][0], lo1 = bd.lo[q][1], lo2 = bd.lo[q][2];
  const int w0 = bd.hi[q][0] - lo0 + 1, w1 = bd.hi[q][1] - lo1 + 1, w2 = bd.hi[q][2] - lo2 + 1;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)w0 * w1 * w2) return;
  const int n3[3] = {lo0 + (int)(t % w0), lo1 + (int)((t / w0) % w1), lo2 + (int)(t / ((int64_t)w0 * w1))};
  long long sum = 0;
#pragma unroll
  for (int f = 0; f < 6; f++) {
    const int d = f >> 1, e1 = d == 0 ? 1 : 0, e2 = d == 2 ? 1 : 2;
    if (n3[d] != ((f & 1) ? bd.hi[q][d] : bd.lo[q][d])) continue;
    const int ext1 = bd.hi[q][e1] - bd.lo[q][e1], ext2 = bd.hi[q][e2] - bd.lo[q][e2];
    const int a = n3[e1] - bd.lo[q][e1], b = n3[e2] - bd.lo[q][e2];  // node (a, b) of the face
    for (int v = b - 1; v <= b; v++)
      for (int u = a - 1; u <= a; u++)
        if (u >= 0 && v >= 0 && u < ext1 && v < ext2)
          sum += (long long)surf[bd.off[q][f] + u + (int64_t)ext1 * v];
  }
  if (sum != 0) {
    const int64_t x = fr.at(0, n3[0], n3[1], n3[2]);
    rhobk[x] = rhobk[x] + qs * 0.25 * (double)sum;
  }
}

// rho(0:n) += rhobk(0:n), or = rhobk(0:n) (charge.F90:440-448).
__global__ void k_add_background(double* __restrict__ rho, const double* __restrict__ rhobk, FieldDesc fr, int nx,
                                 int ny, int nz, int replace) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= fr.size()) return;
  const int64_t ex = fr.ex, ey = fr.ey;
  const int i = (int)(e % ex) + fr.lo, j = (int)((e / ex) % ey) + fr.lo, k = (int)(e / (ex * ey)) + fr.lo;
  if (i < 0 || j < 0 || k < 0 || i > nx || j > ny || k > nz) return;
  rho[e] = replace ? rhobk[e] : rho[e] + rhobk[e];
}
