// fx_adjoint.cuh -- reverse-mode (adjoint) step of the FP32 form on a
// periodic grid (included by fx.cu after fx_push.cuh).
//
// One CTA per (tile, species) region of the thread-major layout, one thread
// per column as in the push.  For the particle state S_n of step n and the
// adjoint (lambda_x, lambda_v) of S_{n+1}, each particle recomputes its
// forward step (trilinear gather of the node fields, Buneman-Boris, move,
// zigzag relay points) and runs it backwards:
//   zigzag     dS/da, dS/db of S = sum_nodes g . J_particle, g = dL/dJ of
//              this step on the nodes (2 Jx on the probe nodes)
//   move       a = b + v_{n+1} ustep: lambda_v += ustep lambda_a,
//              lambda_b += lambda_a
//   Boris      the rotation transposed term by term -> lambda_v_n,
//              lambda_E, lambda_B at the particle
//   gather     w_c lambda_E, w_c lambda_B added to the node-field gradients
//              (per-thread FP32 run sums in registers, added into an FP64
//              shared-memory box when the thread's cell changes, then FP64
//              global atomics: the gradient sums over particles and steps run
//              in FP64);
//              sum_c grad(w_c) (E_c . lambda_E + B_c . lambda_B) added to
//              lambda_x
// The same formulas in FP64 are the CPU checker (oracle/adjoint.cpp).

struct AdjArgs {
  const float4* pos;
  const float* vx;
  const float* vy;
  const float* vz;
  float* lx;                    // adjoint of the position (x, y, z), written
  float* ly;
  float* lz;
  float* lvx;                   // adjoint of the velocity, written
  float* lvy;
  float* lvz;
  // lambda of the next state, read: the arrays above (in place) or, across
  // a re-sort, the next state's arrays at slot off + fwd[slot - off] (fwd:
  // the sort's old slot -> new slot, per species region)
  const float* slx;
  const float* sly;
  const float* slz;
  const float* slvx;
  const float* slvy;
  const float* slvz;
  const uint32_t* fwd;
  const int64_t* tile_start;
  const int64_t* tile_pad;
  int64_t off[EMSESG_ISPEC];
  float qmp[EMSESG_ISPEC], q[EMSESG_ISPEC];
  float us, rustep;
  const float4* __restrict__ f0;  // node fields (nodes 0..n per axis)
  const float4* __restrict__ f1;
  const float* __restrict__ g;    // dL/dJ per unique node, 3 components
  double* gE;                     // node-field gradients per unique node, 3 + 3 (FP64 sums)
  double* gB;
  Geo geo;
  int64_t ntiles;
};

__device__ __forceinline__ int64_t unique_node(const Geo& G, int i, int j, int k) {
  i %= G.nx; if (i < 0) i += G.nx;
  j %= G.ny; if (j < 0) j += G.ny;
  k %= G.nz; if (k < 0) k += G.nz;
  return (int64_t)i + (int64_t)G.nx * ((int64_t)j + (int64_t)G.ny * k);
}

template <int B>
struct AdjBox {
  const int* o;
  const float* gs;  // box g, 3 per node
  const Geo* G;
  const float* gglob;
  __device__ float g(int comp, int i, int j, int k) const {
    const int li = i - o[0], lj = j - o[1], lk = k - o[2];
    if ((unsigned)li < (unsigned)B && (unsigned)lj < (unsigned)B && (unsigned)lk < (unsigned)B)
      return gs[3 * ((lk * B + lj) * B + li) + comp];
    return gglob[3 * unique_node(*G, i, j, k) + comp];
  }
};

// dS/da and dS/db (local coordinates of cell b) of the zigzag deposit.
template <int B>
__device__ __forceinline__ void zigzag_adj(const AdjBox<B>& bx, const int (&cb)[3], const int (&ca)[3],
                                           const float (&bl)[3], const float (&al)[3], float q, float rustep,
                                           float (&dSda)[3], float (&dSdb)[3]) {
  float r[3], drd[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const bool same = ca[k] == cb[k];
    r[k] = same ? 0.5f * (al[k] + bl[k]) : (ca[k] > cb[k] ? 1.0f : 0.0f);
    drd[k] = same ? 0.5f : 0.0f;
    dSda[k] = 0.f;
    dSdb[k] = 0.f;
  }
#pragma unroll
  for (int s = 0; s < 2; s++) {
    float F[3], d[3], dFa[3], dFb[3], dda[3], ddb[3];
    int cell[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      if (s == 0) {
        F[k] = (r[k] - bl[k]) * rustep;
        d[k] = 0.5f * (r[k] + bl[k]);
        dFa[k] = drd[k] * rustep; dFb[k] = (drd[k] - 1.0f) * rustep;
        dda[k] = 0.5f * drd[k]; ddb[k] = 0.5f * (drd[k] + 1.0f);
        cell[k] = cb[k];
      } else {
        const float sh = (float)(ca[k] - cb[k]);
        F[k] = (al[k] - r[k]) * rustep;
        d[k] = 0.5f * (al[k] + r[k]) - sh;
        dFa[k] = (1.0f - drd[k]) * rustep; dFb[k] = -drd[k] * rustep;
        dda[k] = 0.5f * (1.0f + drd[k]); ddb[k] = 0.5f * drd[k];
        cell[k] = ca[k];
      }
    }
#pragma unroll
    for (int comp = 0; comp < 3; comp++) {
      const int p1 = comp == 0 ? 1 : 0, p2 = comp == 2 ? 1 : 2;
      float Gv = 0.f, dG1 = 0.f, dG2 = 0.f;
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const int u = e & 1, v = e >> 1;
        int nd[3] = {cell[0], cell[1], cell[2]};
        nd[p1] += u;
        nd[p2] += v;
        const float W1 = u ? d[p1] : 1.0f - d[p1], W2 = v ? d[p2] : 1.0f - d[p2];
        const float gn = bx.g(comp, nd[0], nd[1], nd[2]);
        Gv += gn * W1 * W2;
        dG1 += gn * (u ? 1.0f : -1.0f) * W2;
        dG2 += gn * W1 * (v ? 1.0f : -1.0f);
      }
      dSda[comp] += q * Gv * dFa[comp];
      dSdb[comp] += q * Gv * dFb[comp];
      dSda[p1] += q * F[comp] * dG1 * dda[p1];
      dSdb[p1] += q * F[comp] * dG1 * ddb[p1];
      dSda[p2] += q * F[comp] * dG2 * dda[p2];
      dSdb[p2] += q * F[comp] * dG2 * ddb[p2];
    }
  }
}

__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 add3(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 mul3(float s, float3 a) { return f3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
  return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

// Threads of a reverse-step CTA: a row of more than 512 slots is taken in
// two column passes by half as many threads (whole warps), so that the
// reverse step keeps its registers (the push's wide rows cap them at 80).
constexpr int ADJ_THREADS = PUSH_THREADS > 512 ? (PUSH_THREADS / 2 + 31) / 32 * 32 : PUSH_THREADS;

template <int T>
__global__ void __launch_bounds__(ADJ_THREADS, 1) k_fx_adjoint(AdjArgs a) {
  constexpr int B = T + 2 * PG + 1;
  constexpr int NF = B * B * B;
  extern __shared__ __align__(16) float4 adj_smem[];
  float4* sf0 = adj_smem;
  float4* sf1 = sf0 + NF;
  double* sgr = reinterpret_cast<double*>(sf1 + NF);  // 6 per node: dE (3), dB (3), FP64
  float* sg = reinterpret_cast<float*>(sgr + 6 * NF);  // 3 per node
  const Geo& G = a.geo;
  const int is = blockIdx.y, t = blockIdx.x, tid = threadIdx.x;
  const int64_t* ts = a.tile_start + (int64_t)is * (a.ntiles + 1);
  const int64_t n = ts[t + 1] - ts[t];
  if (n <= 0) return;
  const int L = (int)((n + PUSH_THREADS - 1) / PUSH_THREADS);
  const int64_t slot0 = a.off[is] + a.tile_pad[(int64_t)is * (a.ntiles + 1) + t];
  const int tx = t % G.nt[0], ty = (t / G.nt[0]) % G.nt[1], tz = t / (G.nt[0] * G.nt[1]);
  const int o[3] = {tx * G.t[0] - PG, ty * G.t[1] - PG, tz * G.t[2] - PG};
  const int64_t sy = G.nx + 1, sz = (int64_t)(G.nx + 1) * (G.ny + 1);
  bool anyg = false;
  for (int e = tid; e < NF; e += ADJ_THREADS) {
    const int li = e % B, lj = (e / B) % B, lk = e / (B * B);
    const int gi = o[0] + li, gj = o[1] + lj, gk = o[2] + lk;
    float4 p = make_float4(0.f, 0.f, 0.f, 0.f), q = p;
    if (gi >= 0 && gj >= 0 && gk >= 0 && gi <= G.nx && gj <= G.ny && gk <= G.nz) {
      const int64_t gn = gi + sy * gj + sz * gk;
      p = __ldg(&a.f0[gn]);
      q = __ldg(&a.f1[gn]);
    }
    sf0[e] = p;
    sf1[e] = q;
    const int64_t un = unique_node(G, gi, gj, gk);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      sg[3 * e + c] = a.g[3 * un + c];
      anyg = anyg || sg[3 * e + c] != 0.f;
    }
#pragma unroll
    for (int c = 0; c < 6; c++) sgr[6 * e + c] = 0.0;
  }
  // dL/dJ is zero on every node of most boxes (the loss sees a probe region
  // only): their particles' zigzag terms are zero and are skipped
  anyg = __syncthreads_or(anyg) != 0;
  const AdjBox<B> bx{o, sg, &G, a.g};
  // the node-field gradient of the thread's current run (its particles of
  // one cell), 6 values for each of the 8 corners, in registers; added into
  // sgr when the run ends, so the shared atomics go per run, not per particle
  float pacc[48];
#pragma unroll
  for (int q = 0; q < 48; q++) pacc[q] = 0.f;
  int runbase = -1;  // box index of the run cell's first corner
  auto flush = [&]() {
    if (runbase < 0) return;
#pragma unroll
    for (int c = 0; c < 8; c++) {
      const int e = runbase + (c >> 2) * B * B + ((c >> 1) & 1) * B + (c & 1);
#pragma unroll
      for (int q = 0; q < 6; q++) {
        if (pacc[6 * c + q] != 0.f) atomicAdd(&sgr[6 * e + q], (double)pacc[6 * c + q]);
        pacc[6 * c + q] = 0.f;
      }
    }
  };
  const float qmp = a.qmp[is], qq = a.q[is], us = a.us, rustep = a.rustep;
  // the thread's columns, one pass each (a run never spans two columns)
  for (int col = tid; col < PUSH_THREADS; col += ADJ_THREADS) {
  for (int r = 0; r < L; r++) {
    const int64_t m = slot0 + (int64_t)r * PUSH_THREADS + col;
    const float4 ps = a.pos[m];
    const uint32_t cell = (uint32_t)__float_as_int(ps.w);
    if (cell == DEAD) continue;
    // lambda of the next state, loaded first: its latency hides behind the
    // recompute
    const int64_t mn = a.fwd ? a.off[is] + (int64_t)a.fwd[m] : m;  // the slot of the next state
    const float lnx = a.slx[mn], lny = a.sly[mn], lnz = a.slz[mn];
    const float lnvx = a.slvx[mn], lnvy = a.slvy[mn], lnvz = a.slvz[mn];
    int cb[3];
    unpack(G, cell, cb[0], cb[1], cb[2]);
    const float bl[3] = {ps.x, ps.y, ps.z};
    const float3 v0 = f3(a.vx[m], a.vy[m], a.vz[m]);
    const int li = cb[0] - o[0], lj = cb[1] - o[1], lk = cb[2] - o[2];
    const bool inb = (unsigned)li < (unsigned)(B - 1) && (unsigned)lj < (unsigned)(B - 1) && (unsigned)lk < (unsigned)(B - 1);
    const int e0 = (lk * B + lj) * B + li;  // box index of corner 0 (in the box)
    // trilinear weights, corner c = di + 2 dj + 4 dk
    float wc[8];
#pragma unroll
    for (int c = 0; c < 8; c++) {
      const int di = c & 1, dj = (c >> 1) & 1, dk = c >> 2;
      const float X = di ? bl[0] : 1.0f - bl[0], Y = dj ? bl[1] : 1.0f - bl[1], Z = dk ? bl[2] : 1.0f - bl[2];
      wc[c] = X * Y * Z;
    }
    // forward recompute: gather
    float3 E = f3(0.f, 0.f, 0.f), Bf = E;
    if (inb) {
#pragma unroll
      for (int c = 0; c < 8; c++) {
        const int e = e0 + (c >> 2) * B * B + ((c >> 1) & 1) * B + (c & 1);
        const float4 cp = sf0[e], cq = sf1[e];
        E = add3(E, mul3(wc[c], f3(cp.x, cp.y, cp.z)));
        Bf = add3(Bf, mul3(wc[c], f3(cp.w, cq.x, cq.y)));
      }
    } else {
#pragma unroll 1
      for (int c = 0; c < 8; c++) {
        const int di = c & 1, dj = (c >> 1) & 1, dk = c >> 2;
        const float X = di ? bl[0] : 1.0f - bl[0], Y = dj ? bl[1] : 1.0f - bl[1], Z = dk ? bl[2] : 1.0f - bl[2];
        const float w = X * Y * Z;
        const int64_t gn = (cb[0] + di) + sy * (cb[1] + dj) + sz * (cb[2] + dk);
        const float4 cp = __ldg(&a.f0[gn]), cq = __ldg(&a.f1[gn]);
        E = add3(E, mul3(w, f3(cp.x, cp.y, cp.z)));
        Bf = add3(Bf, mul3(w, f3(cp.w, cq.x, cq.y)));
      }
    }
    const float3 ee = mul3(qmp, E), tt = mul3(qmp, Bf);
    const float sfac = 2.0f / (1.0f + dot3(tt, tt));
    const float3 uu = add3(v0, ee);
    const float3 ww = add3(uu, cross3(uu, tt));
    const float3 cc = cross3(ww, tt);
    const float3 pp = add3(uu, mul3(sfac, cc));
    const float3 vn = add3(pp, ee);
    const float vnv[3] = {vn.x, vn.y, vn.z};
    float al[3];
    int ca[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      al[k] = bl[k] + vnv[k] * us;
      ca[k] = cb[k] + (int)floorf(al[k]);
    }
    float dSda[3] = {0.f, 0.f, 0.f}, dSdb[3] = {0.f, 0.f, 0.f};
    const bool ina = (unsigned)(ca[0] - o[0]) < (unsigned)(B - 1) && (unsigned)(ca[1] - o[1]) < (unsigned)(B - 1) &&
                     (unsigned)(ca[2] - o[2]) < (unsigned)(B - 1);
    if (anyg || !inb || !ina) zigzag_adj<B>(bx, cb, ca, bl, al, qq, rustep, dSda, dSdb);
    // move: a = b + vnew * ustep
    const float3 la = f3(lnx + dSda[0], lny + dSda[1], lnz + dSda[2]);
    const float3 lvn = add3(f3(lnvx, lnvy, lnvz), mul3(us, la));
    float3 lb = add3(f3(dSdb[0], dSdb[1], dSdb[2]), la);
    // Boris, reversed
    float3 le = lvn;
    const float3 lp = lvn;
    float3 lu = lp;
    const float ls = dot3(lp, cc);
    const float3 lc = mul3(sfac, lp);
    const float3 lw = cross3(tt, lc);
    float3 lt = cross3(lc, ww);
    lu = add3(add3(lu, lw), cross3(tt, lw));
    lt = add3(lt, cross3(lw, uu));
    lt = add3(lt, mul3(-ls * sfac * sfac, tt));
    le = add3(le, lu);
    const float3 lE = mul3(qmp, le), lB = mul3(qmp, lt);
    // gather, reversed: the node-field gradients w_c lambda, and to lambda_b
    // the gradient of sum_c w_c s_c, s_c = (E_c, B_c) . (lambda_E, lambda_B)
    if (inb) {
      if (e0 != runbase) {
        flush();
        runbase = e0;
      }
      float sc[8];
#pragma unroll
      for (int c = 0; c < 8; c++) {
        const int e = e0 + (c >> 2) * B * B + ((c >> 1) & 1) * B + (c & 1);
        const float4 cp = sf0[e], cq = sf1[e];
        sc[c] = cp.x * lE.x + cp.y * lE.y + cp.z * lE.z + cp.w * lB.x + cq.x * lB.y + cq.y * lB.z;
        const float gv[6] = {lE.x, lE.y, lE.z, lB.x, lB.y, lB.z};
#pragma unroll
        for (int q = 0; q < 6; q++) pacc[6 * c + q] = fmaf(wc[c], gv[q], pacc[6 * c + q]);
      }
      // trilinear interpolation of sc in x, then y, then z, with the
      // derivatives carried along
      float dx[4], ax[4];
#pragma unroll
      for (int h = 0; h < 4; h++) {
        dx[h] = sc[2 * h + 1] - sc[2 * h];
        ax[h] = fmaf(bl[0], dx[h], sc[2 * h]);
      }
      float ey[2], cy[2], bxy[2];
#pragma unroll
      for (int k = 0; k < 2; k++) {
        ey[k] = ax[2 * k + 1] - ax[2 * k];
        cy[k] = fmaf(bl[1], ey[k], ax[2 * k]);
        bxy[k] = fmaf(bl[1], dx[2 * k + 1] - dx[2 * k], dx[2 * k]);
      }
      lb.x += fmaf(bl[2], bxy[1] - bxy[0], bxy[0]);
      lb.y += fmaf(bl[2], ey[1] - ey[0], ey[0]);
      lb.z += cy[1] - cy[0];
    } else {
#pragma unroll 1
      for (int c = 0; c < 8; c++) {
        const int di = c & 1, dj = (c >> 1) & 1, dk = c >> 2;
        const float X = di ? bl[0] : 1.0f - bl[0], Y = dj ? bl[1] : 1.0f - bl[1], Z = dk ? bl[2] : 1.0f - bl[2];
        const float dX = di ? 1.0f : -1.0f, dY = dj ? 1.0f : -1.0f, dZ = dk ? 1.0f : -1.0f;
        const float w = X * Y * Z;
        const int64_t gn = (cb[0] + di) + sy * (cb[1] + dj) + sz * (cb[2] + dk);
        const float4 cp = __ldg(&a.f0[gn]), cq = __ldg(&a.f1[gn]);
        const float sdot = cp.x * lE.x + cp.y * lE.y + cp.z * lE.z + cp.w * lB.x + cq.x * lB.y + cq.y * lB.z;
        lb = add3(lb, mul3(sdot, f3(dX * Y * Z, X * dY * Z, X * Y * dZ)));
        const float gv[6] = {w * lE.x, w * lE.y, w * lE.z, w * lB.x, w * lB.y, w * lB.z};
        const int64_t un = unique_node(G, cb[0] + di, cb[1] + dj, cb[2] + dk);
#pragma unroll
        for (int q = 0; q < 3; q++) {
          atomicAdd(&a.gE[3 * un + q], (double)gv[q]);
          atomicAdd(&a.gB[3 * un + q], (double)gv[3 + q]);
        }
      }
    }
    a.lx[m] = lb.x;
    a.ly[m] = lb.y;
    a.lz[m] = lb.z;
    a.lvx[m] = lu.x;
    a.lvy[m] = lu.y;
    a.lvz[m] = lu.z;
  }
  flush();
  runbase = -1;
  }  // column passes
  __syncthreads();
  for (int e = tid; e < NF; e += ADJ_THREADS) {
    const int li = e % B, lj = (e / B) % B, lk = e / (B * B);
    const int gi = o[0] + li, gj = o[1] + lj, gk = o[2] + lk;
    if (gi < 0 || gj < 0 || gk < 0 || gi > G.nx || gj > G.ny || gk > G.nz) continue;
    const int64_t un = unique_node(G, gi, gj, gk);
#pragma unroll
    for (int q = 0; q < 3; q++) {
      const double vE = sgr[6 * e + q], vB = sgr[6 * e + 3 + q];
      if (vE != 0.0) atomicAdd(&a.gE[3 * un + q], vE);
      if (vB != 0.0) atomicAdd(&a.gB[3 * un + q], vB);
    }
  }
}

inline int fx_adjoint_smem(int tmax) {
  const int B = fx_box_tile(tmax) + 2 * PG + 1;
  const int nf = B * B * B;
  return nf * (int)(2 * sizeof(float4) + 6 * sizeof(double) + 3 * sizeof(float));
}

// The forward map of a sort from its inverse (inv[new slot] = old slot,
// region-relative, DEAD for empty slots): fwd[old slot] = new slot, so that
// the reverse step of S_n (old layout) reads the lambda of S_{n+1} (new
// layout) in place of a separate unsort of lambda.
__global__ void k_adj_fwd(const uint32_t* __restrict__ inv, int64_t n, uint32_t* fwd) {
  const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  const uint32_t s = inv[m];
  if (s != DEAD) fwd[s] = (uint32_t)m;
}

// A sort of the forward pass applied again from its kept map (inv[new slot]
// = old slot, region-relative, DEAD for an empty slot): the records of the
// new layout gathered from the old one, empty slots as the sort leaves them.
// The recompute of a segment repeats its sorts this way instead of sorting.
__global__ void k_adj_apply(const uint32_t* __restrict__ inv, int64_t n, const float4* __restrict__ pos,
                            const float* __restrict__ vx, const float* __restrict__ vy, const float* __restrict__ vz,
                            float4* __restrict__ pos2, float* __restrict__ vx2, float* __restrict__ vy2,
                            float* __restrict__ vz2) {
  const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  const uint32_t s = inv[m];
  float4 p = make_float4(0.f, 0.f, 0.f, __int_as_float((int)DEAD));
  float a = 0.f, b = 0.f, c = 0.f;
  if (s != DEAD) {
    p = pos[s];
    a = vx[s];
    b = vy[s];
    c = vz[s];
  }
  pos2[m] = p;
  vx2[m] = a;
  vy2[m] = b;
  vz2[m] = c;
}

__device__ __forceinline__ bool in_probe(const Geo& G, int64_t un, int3 lo, int3 hi, int& i, int& j, int& k) {
  i = (int)(un % G.nx);
  j = (int)((un / G.nx) % G.ny);
  k = (int)(un / ((int64_t)G.nx * G.ny));
  return i >= lo.x && i < hi.x && j >= lo.y && j < hi.y && k >= lo.z && k < hi.z;
}

// The loss of one step, sum over the probe nodes of aj_x^2 (aj: the folded
// FP64 current), and, when jx_keep is given, the probe Jx of the step.
__global__ void k_adj_probe(const double* __restrict__ aj, FieldDesc fj, Geo G, int3 lo, int3 hi, double* loss,
                            float* jx_keep) {
  const int64_t un = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (un >= (int64_t)G.nx * G.ny * G.nz) return;
  int i, j, k;
  if (!in_probe(G, un, lo, hi, i, j, k)) {
    if (jx_keep) jx_keep[un] = 0.f;
    return;
  }
  const double jx = aj[fj.at(0, i, j, k)];
  if (loss) atomicAdd(loss, jx * jx);
  if (jx_keep) jx_keep[un] = (float)jx;
}

// g = dL/dJ of one step: 2 Jx on the probe nodes, 0 elsewhere.
__global__ void k_adj_g(const float* __restrict__ jx, int64_t nn, float* g) {
  const int64_t un = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (un >= nn) return;
  g[3 * un] = 2.0f * jx[un];
  g[3 * un + 1] = 0.f;
  g[3 * un + 2] = 0.f;
}

// lambda_v of the start state (thread-major regions) in canonical order
// (tile-major sorted ranks): out[(rank0 + q) * 3 + c].
__global__ void k_adj_canonical(const float* __restrict__ lvx, const float* __restrict__ lvy,
                                const float* __restrict__ lvz, const int64_t* __restrict__ ts,
                                const int64_t* __restrict__ tp, int64_t rank0, double* out) {
  const int t = blockIdx.x, tid = threadIdx.x;
  const int64_t n = ts[t + 1] - ts[t];
  if (n <= 0) return;
  const int L = (int)((n + PUSH_THREADS - 1) / PUSH_THREADS);
  for (int r = 0; r < L; r++) {
    const int64_t q = (int64_t)tid * L + r;
    if (q >= n) continue;
    const int64_t m = tp[t] + (int64_t)r * PUSH_THREADS + tid;
    double* o = out + 3 * (rank0 + ts[t] + q);
    o[0] = lvx[m];
    o[1] = lvy[m];
    o[2] = lvz[m];
  }
}
