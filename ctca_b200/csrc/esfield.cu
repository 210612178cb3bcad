// esfield.cu -- the electrostatic field step of the reference on the device:
// esfld1(0) with poisson(3) (the FFT solution of the discrete Poisson
// equation), the guards of phi, esfld2 (E on its staggered positions from
// phi) and poichk (the residual of the discrete equation), for every
// field boundary of the Poisson solve (mtd_vbnd: 0 periodic, 1 phi = 0 on the
// faces, 2 Neumann).  FP64 throughout, like the reference's field arrays.
//
// poisson (src/field/poisson/poissn.F90:216-470 with the periodic set-up of
// src/field/poisson/inifft.F90:389-470) transforms rho on the nodes 0..n-1 of
// every axis with FFTW's real-to-halfcomplex DFT along x, y and z, divides
// every coefficient by mfactor * (kmod_x + kmod_y + kmod_z), where
// kmod(m) = (2 sin(pi m / n) / dr)^2 is the eigenvalue of the 3-point
// -d2/dx2 at the mode's frequency and mfactor = nx ny nz undoes the
// unnormalised transforms, sets the mean mode to zero, and transforms back.
// The products of cosines and sines those separable transforms expand into
// are eigenfunctions of the 7-point Laplacian with the same eigenvalues as
// the complex exponentials, so the same solution -- the zero-mean phi with
// rho + (sum of the six neighbours of phi) - 6 phi = mean(rho) on every
// node -- comes out of one complex real-to-complex transform (cuFFT D2Z /
// Z2D) divided by the same eigenvalues; the two differ by the rounding of
// the transforms.  That is the path when every axis is periodic.
//
// With a face on some axis (inifft.F90:409-424: mtd_vbnd 1 solves the nodes
// 1..n-1 with FFTW_RODFT00, a type-1 DST; 2 the nodes 0..n with
// FFTW_REDFT00, a type-1 DCT; both with kmod(i) = 2 (1 - cos(i pi / n)) / dr^2
// and a factor 2n in mfactor) the transforms run axis by axis, as the
// reference's r2r transforms do: every line of the axis is laid out in a
// complex buffer -- as it is (periodic), or extended to 2n points oddly
// (0, x, 0, -reversed x) for the DST or evenly (x, reversed inner x) for the
// DCT -- one batched complex FFT (cuFFT Z2Z) transforms all lines, and the
// real r2r output is read back (the halfcomplex layout, -Im for the DST,
// Re for the DCT).  Neumann faces first add their boundary values to rho
// (poissn.F90:76-127), and esfld2 then copies (mtd_vbnd 1) or negates
// (mtd_vbnd 2) the normal E component at -1 and n from 0 and n-1
// (esfild.F90:368-435).
#include <algorithm>
#include <cmath>
#include <cufft.h>

#include "common.cuh"

namespace emsesg {

namespace {

constexpr int ES_BLOCK = 256;

inline unsigned es_blocks(int64_t n) { return (unsigned)((n + ES_BLOCK - 1) / ES_BLOCK); }

// rho on the nodes 0..n-1 (node n is node 0 on a periodic axis) -> r[k][j][i]
__global__ void k_es_pack(const double* __restrict__ rho, FieldDesc fr, int nx, int ny, int nz,
                          double* __restrict__ r) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)nx * ny * nz) return;
  const int i = (int)(t % nx), j = (int)((t / nx) % ny), k = (int)(t / ((int64_t)nx * ny));
  r[t] = rho[fr.at(0, i, j, k)];
}

// The spectrum of r (nz x ny x (nx/2+1) complex) divided by
// N * (lx[i] + ly[j] + lz[k]) (poissn.F90:418-430); the mean mode becomes 0.
__global__ void k_es_divide(cufftDoubleComplex* __restrict__ c, const double* __restrict__ lx,
                            const double* __restrict__ ly, const double* __restrict__ lz, int nxh, int ny, int nz,
                            double mfactor) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)nxh * ny * nz) return;
  const int i = (int)(t % nxh), j = (int)((t / nxh) % ny), k = (int)(t / ((int64_t)nxh * ny));
  const double divisor = (lx[i] + ly[j] + lz[k]) * mfactor;
  cufftDoubleComplex v = c[t];
  if (divisor != 0.0) {
    v.x = v.x / divisor;
    v.y = v.y / divisor;
  } else {
    v.x = 0.0;
    v.y = 0.0;
  }
  c[t] = v;
}

// The solution on the nodes 0..n-1 -> phi on -1..n+1 with the periodic
// guards of poissn.F90:686-710: phi(-1) = phi(n-1), phi(n) = phi(0),
// phi(n+1) = phi(1) on every axis.
__global__ void k_es_unpack(const double* __restrict__ p, double* __restrict__ phi, FieldDesc fp, int nx, int ny,
                            int nz) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int ex = nx + 3, ey = ny + 3, ez = nz + 3;
  if (t >= (int64_t)ex * ey * ez) return;
  const int i = (int)(t % ex) - 1, j = (int)((t / ex) % ey) - 1, k = (int)(t / ((int64_t)ex * ey)) - 1;
  const int si = (i + nx) % nx, sj = (j + ny) % ny, sk = (k + nz) % nz;
  phi[fp.at(0, i, j, k)] = p[si + (int64_t)nx * (sj + (int64_t)ny * sk)];
}

// esfld2 (src/field/esfild.F90:351-366): EX..EZ cleared, then
// EX(i,j,k) = (phi(i,j,k) - phi(i+1,j,k)) * mltstp on i = -1..n, j, k = 0..n,
// and the same along y and z.  One thread per eb node; the B components are
// left as they are.
__global__ void k_es_efield(const double* __restrict__ phi, FieldDesc fp, double* __restrict__ eb, FieldDesc fe,
                            int nx, int ny, int nz, double mlt, int tx, int ty, int tz) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)fe.ex * fe.ey * fe.ez) return;
  const int i = (int)(t % fe.ex) + fe.lo, j = (int)((t / fe.ex) % fe.ey) + fe.lo,
            k = (int)(t / ((int64_t)fe.ex * fe.ey)) + fe.lo;
  const bool jk = j >= 0 && j <= ny && k >= 0 && k <= nz;
  const bool ik = i >= 0 && i <= nx && k >= 0 && k <= nz;
  const bool ij = i >= 0 && i <= nx && j >= 0 && j <= ny;
  const double p = (i <= nx + 1 && j <= ny + 1 && k <= nz + 1) ? phi[fp.at(0, i, j, k)] : 0.0;
  double ex = (jk && i <= nx) ? (p - phi[fp.at(0, i + 1, j, k)]) * mlt : 0.0;
  double ey = (ik && j <= ny) ? (p - phi[fp.at(0, i, j + 1, k)]) * mlt : 0.0;
  double ez = (ij && k <= nz) ? (p - phi[fp.at(0, i, j, k + 1)]) * mlt : 0.0;
  // a face: the normal component at -1 / n is the one at 0 / n-1, copied
  // (mtd_vbnd 1) or negated (2)
  if (tx != 0 && jk && (i == -1 || i == nx)) {
    const int a = i == -1 ? 0 : nx - 1;
    ex = (tx == 1 ? 1.0 : -1.0) * ((phi[fp.at(0, a, j, k)] - phi[fp.at(0, a + 1, j, k)]) * mlt);
  }
  if (ty != 0 && ik && (j == -1 || j == ny)) {
    const int a = j == -1 ? 0 : ny - 1;
    ey = (ty == 1 ? 1.0 : -1.0) * ((phi[fp.at(0, i, a, k)] - phi[fp.at(0, i, a + 1, k)]) * mlt);
  }
  if (tz != 0 && ij && (k == -1 || k == nz)) {
    const int a = k == -1 ? 0 : nz - 1;
    ez = (tz == 1 ? 1.0 : -1.0) * ((phi[fp.at(0, i, j, a)] - phi[fp.at(0, i, j, a + 1)]) * mlt);
  }
  eb[fe.at(0, i, j, k)] = ex;
  eb[fe.at(1, i, j, k)] = ey;
  eb[fe.at(2, i, j, k)] = ez;
}

// poichk (poissn.F90:937-948): the sum of squares of
// rho + (phi(i-1) + phi(i+1) + phi(j-1) + phi(j+1) + phi(k-1) + phi(k+1)) - 6 phi
// over its loop's nodes (from the first solved node, cx x cy x cz of them),
// in the order of the terms there; one atomic per block.
__global__ void k_es_poichk(const double* __restrict__ rho, FieldDesc fr, const double* __restrict__ phi,
                            FieldDesc fp, int x0, int y0, int z0, int cx, int cy, int cz, double* __restrict__ sum) {
  __shared__ double part[ES_BLOCK / 32];
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double d2 = 0.0;
  if (t < (int64_t)cx * cy * cz) {
    const int i = x0 + (int)(t % cx), j = y0 + (int)((t / cx) % cy), k = z0 + (int)(t / ((int64_t)cx * cy));
    const double drho = rho[fr.at(0, i, j, k)] +
                        (phi[fp.at(0, i - 1, j, k)] + phi[fp.at(0, i + 1, j, k)] + phi[fp.at(0, i, j - 1, k)] +
                         phi[fp.at(0, i, j + 1, k)] + phi[fp.at(0, i, j, k - 1)] + phi[fp.at(0, i, j, k + 1)]) -
                        6.0 * phi[fp.at(0, i, j, k)];
    d2 = drho * drho;
  }
  for (int o = 16; o > 0; o >>= 1) d2 += __shfl_down_sync(0xffffffffu, d2, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = d2;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < ES_BLOCK / 32; w++) s += part[w];
    atomicAdd(sum, s);
  }
}

// ---- any field boundary: axis by axis
struct EsGeo {
  int n[3];   // cells per axis
  int t[3];   // mtd_vbnd
  int lo[3];  // first solved node
  int m[3];   // solved nodes
};
struct EsBc {
  double v[6];  // boundary_conditions(side, axis) * rene, [2 axis + side]
};

// rho on the solved nodes, with the Neumann faces' boundary values added
// axis by axis as poissn.F90:76-127 adds them (x, then y, then z planes).
__global__ void k_es_pack_w(const double* __restrict__ rho, FieldDesc fr, EsGeo G, EsBc bc, double* __restrict__ w) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)G.m[0] * G.m[1] * G.m[2]) return;
  const int nd[3] = {G.lo[0] + (int)(t % G.m[0]), G.lo[1] + (int)((t / G.m[0]) % G.m[1]),
                     G.lo[2] + (int)(t / ((int64_t)G.m[0] * G.m[1]))};
  double v = rho[fr.at(0, nd[0], nd[1], nd[2])];
  for (int d = 0; d < 3; d++) {
    if (G.t[d] != 2) continue;
    if (nd[d] == 0) v = v - bc.v[2 * d] * 2.0;
    if (nd[d] == G.n[d]) v = v + bc.v[2 * d + 1] * 2.0;
  }
  w[t] = v;
}

// w index of (position u along axis a, line l): l runs over the other two
// axes, the lower one fastest.
__device__ __forceinline__ int64_t es_widx(const EsGeo& G, int a, int64_t l, int u) {
  const int p = a == 0 ? 1 : 0, q = a == 2 ? 1 : 2;
  int id[3];
  id[a] = u;
  id[p] = (int)(l % G.m[p]);
  id[q] = (int)(l / G.m[p]);
  return id[0] + (int64_t)G.m[0] * (id[1] + (int64_t)G.m[1] * id[2]);
}

// Line transforms of axis a (kind 0: R2HC, 1: HC2R, 2: RODFT00, 3: REDFT00):
// the complex lines of length L the FFT takes ...
__global__ void k_es_line_in(const double* __restrict__ w, EsGeo G, int a, int kind, int L, int64_t lines,
                             cufftDoubleComplex* __restrict__ z) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= lines * L) return;
  const int64_t l = t / L;
  const int u = (int)(t % L), n = G.n[a];
  double re = 0.0, im = 0.0;
  if (kind == 0) {
    re = w[es_widx(G, a, l, u)];
  } else if (kind == 1) {
    // X_0 = h_0, X_k = h_k + i h_(n-k), X_(n/2) = h_(n/2), X_(n-k) = conj(X_k)
    if (u == 0 || 2 * u == n) {
      re = w[es_widx(G, a, l, u)];
    } else if (2 * u < n) {
      re = w[es_widx(G, a, l, u)];
      im = w[es_widx(G, a, l, n - u)];
    } else {
      re = w[es_widx(G, a, l, n - u)];
      im = -w[es_widx(G, a, l, u)];
    }
  } else if (kind == 2) {
    // odd extension over 2n points: (0, x_0..x_(n-2), 0, -x_(n-2)..-x_0)
    if (u >= 1 && u <= n - 1) re = w[es_widx(G, a, l, u - 1)];
    else if (u >= n + 1) re = -w[es_widx(G, a, l, L - u - 1)];
  } else {
    // even extension over 2n points: (x_0..x_n, x_(n-1)..x_1)
    re = w[es_widx(G, a, l, u <= n ? u : L - u)];
  }
  z[t] = make_cuDoubleComplex(re, im);
}

// ... and the real r2r output read back from them.
__global__ void k_es_line_out(const cufftDoubleComplex* __restrict__ z, EsGeo G, int a, int kind, int L,
                              int64_t lines, double* __restrict__ w) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int m = G.m[a], n = G.n[a];
  if (t >= lines * m) return;
  const int64_t l = t / m;
  const int u = (int)(t % m);
  const cufftDoubleComplex* zl = z + l * L;
  double v;
  if (kind == 0) v = 2 * u <= n ? zl[u].x : zl[n - u].y;
  else if (kind == 1) v = zl[u].x;
  else if (kind == 2) v = -zl[u + 1].y;
  else v = zl[u].x;
  w[es_widx(G, a, l, u)] = v;
}

// The coefficients divided by (kmod_x + kmod_y + kmod_z) * mfactor.
__global__ void k_es_divide_w(double* __restrict__ w, const double* __restrict__ lx, const double* __restrict__ ly,
                              const double* __restrict__ lz, EsGeo G, double mfactor) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)G.m[0] * G.m[1] * G.m[2]) return;
  const int i = (int)(t % G.m[0]), j = (int)((t / G.m[0]) % G.m[1]), k = (int)(t / ((int64_t)G.m[0] * G.m[1]));
  const double divisor = (lx[i] + ly[j] + lz[k]) * mfactor;
  w[t] = divisor != 0.0 ? w[t] / divisor : 0.0;
}

// phi on -1..n+1: the solved nodes from w, zero outside them, the periodic
// copies on periodic axes (poissn.F90:672-710).
__global__ void k_es_unpack_w(const double* __restrict__ w, double* __restrict__ phi, FieldDesc fp, EsGeo G) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int ex = G.n[0] + 3, ey = G.n[1] + 3, ez = G.n[2] + 3;
  if (t >= (int64_t)ex * ey * ez) return;
  const int nd[3] = {(int)(t % ex) - 1, (int)((t / ex) % ey) - 1, (int)(t / ((int64_t)ex * ey)) - 1};
  int id[3];
  bool in = true;
  for (int d = 0; d < 3; d++) {
    int x = nd[d];
    if (G.t[d] == 0) x = (x + G.n[d]) % G.n[d];
    id[d] = x - G.lo[d];
    in = in && id[d] >= 0 && id[d] < G.m[d];
  }
  phi[fp.at(0, nd[0], nd[1], nd[2])] = in ? w[id[0] + (int64_t)G.m[0] * (id[1] + (int64_t)G.m[1] * id[2])] : 0.0;
}

// kmod(:, :, 2) of a periodic axis (inifft.F90:392-403) on the complex
// transform's index m: (2 sin(pi i / n) / dr)^2 with i = min(m, n - m), the
// frequency the halfcomplex slot m holds there (dr = 1).
void kmod_periodic(int n, int count, double* out) {
  const double pi = std::acos(-1.0), rn = 1.0 / n, dri = 1.0;
  for (int m = 0; m < count; m++) {
    const int i = m <= n / 2 ? m : n - m;
    double k = 2.0 * std::sin(pi * i * rn) * dri;
    out[m] = k * k;
  }
}

int es_setup(emsesg_ctx* ctx) {
  EsState& s = ctx->es;
  if (s.ready) return EMSESG_OK;
  const emsesg_config& c = ctx->cfg;
  const int nx = c.nx, ny = c.ny, nz = c.nz, nxh = nx / 2 + 1;
  const int64_t n = (int64_t)nx * ny * nz, nh = (int64_t)nxh * ny * nz;
  EMSESG_CUDA(ctx, cudaMalloc(&s.r, n * sizeof(double)));
  EMSESG_CUDA(ctx, cudaMalloc(&s.c, nh * sizeof(cufftDoubleComplex)));
  EMSESG_CUDA(ctx, cudaMalloc(&s.lam, (int64_t)(nxh + ny + nz) * sizeof(double)));
  if (!s.sum) EMSESG_CUDA(ctx, cudaMalloc(&s.sum, sizeof(double)));
  std::vector<double> lam((size_t)(nxh + ny + nz));
  kmod_periodic(nx, nxh, lam.data());
  kmod_periodic(ny, ny, lam.data() + nxh);
  kmod_periodic(nz, nz, lam.data() + nxh + ny);
  EMSESG_CUDA(ctx, cudaMemcpy(s.lam, lam.data(), lam.size() * sizeof(double), cudaMemcpyHostToDevice));
  cufftHandle f = 0, b = 0;
  if (cufftPlan3d(&f, nz, ny, nx, CUFFT_D2Z) != CUFFT_SUCCESS)
    return set_error(ctx, EMSESG_ERR_CUDA, "cufftPlan3d (D2Z %d x %d x %d) failed", nz, ny, nx);
  s.fwd = (int)f;
  s.has_fwd = true;
  if (cufftPlan3d(&b, nz, ny, nx, CUFFT_Z2D) != CUFFT_SUCCESS)
    return set_error(ctx, EMSESG_ERR_CUDA, "cufftPlan3d (Z2D %d x %d x %d) failed", nz, ny, nx);
  s.inv = (int)b;
  s.has_inv = true;
  if (cufftSetStream(f, ctx->stream) != CUFFT_SUCCESS || cufftSetStream(b, ctx->stream) != CUFFT_SUCCESS)
    return set_error(ctx, EMSESG_ERR_CUDA, "cufftSetStream failed");
  s.ready = true;
  return EMSESG_OK;
}

// kmod(:, :, 2) over the solved nodes of an axis with a face
// (inifft.F90:411-414): 2 (1 - cos(i pi / n)) / dr^2, node i from lo.
void kmod_faces(int n, int lo, int count, double* out) {
  const double pi = std::acos(-1.0), dri = 1.0;
  for (int m = 0; m < count; m++) {
    const int i = lo + m;
    out[m] = 2.0 * (1.0 - std::cos(i * pi / n)) * dri * dri;
  }
}

EsGeo es_geo(const emsesg_config& c, const int* t) {
  EsGeo G{};
  const int n[3] = {c.nx, c.ny, c.nz};
  for (int d = 0; d < 3; d++) {
    G.n[d] = n[d];
    G.t[d] = t[d];
    G.lo[d] = t[d] == 1 ? 1 : 0;
    G.m[d] = t[d] == 0 ? n[d] : (t[d] == 1 ? n[d] - 1 : n[d] + 1);
  }
  return G;
}

inline int es_line_len(const EsGeo& G, int a) { return G.t[a] == 0 ? G.n[a] : 2 * G.n[a]; }

void es_free_general(EsState& s) {
  for (int a = 0; a < 3; a++)
    if (s.has_gplan[a]) cufftDestroy((cufftHandle)s.gplan[a]);
  cudaFree(s.w);
  cudaFree(s.z);
  cudaFree(s.glam);
  for (int a = 0; a < 3; a++) {
    s.gplan[a] = 0;
    s.has_gplan[a] = false;
    s.gt[a] = -1;
  }
  s.w = nullptr;
  s.z = nullptr;
  s.glam = nullptr;
}

int es_setup_general(emsesg_ctx* ctx, const int* t) {
  EsState& s = ctx->es;
  if (s.gt[0] == t[0] && s.gt[1] == t[1] && s.gt[2] == t[2]) return EMSESG_OK;
  es_free_general(s);
  const EsGeo G = es_geo(ctx->cfg, t);
  const int64_t nw = (int64_t)G.m[0] * G.m[1] * G.m[2];
  int64_t nz = 0;
  for (int a = 0; a < 3; a++) nz = std::max<int64_t>(nz, nw / G.m[a] * es_line_len(G, a));
  if (!s.sum) EMSESG_CUDA(ctx, cudaMalloc(&s.sum, sizeof(double)));
  EMSESG_CUDA(ctx, cudaMalloc(&s.w, nw * sizeof(double)));
  EMSESG_CUDA(ctx, cudaMalloc(&s.z, nz * sizeof(cufftDoubleComplex)));
  EMSESG_CUDA(ctx, cudaMalloc(&s.glam, (int64_t)(G.m[0] + G.m[1] + G.m[2]) * sizeof(double)));
  std::vector<double> lam((size_t)(G.m[0] + G.m[1] + G.m[2]));
  double* at = lam.data();
  for (int a = 0; a < 3; a++) {
    if (t[a] == 0) kmod_periodic(G.n[a], G.m[a], at);
    else kmod_faces(G.n[a], G.lo[a], G.m[a], at);
    at += G.m[a];
  }
  EMSESG_CUDA(ctx, cudaMemcpy(s.glam, lam.data(), lam.size() * sizeof(double), cudaMemcpyHostToDevice));
  for (int a = 0; a < 3; a++) {
    int L = es_line_len(G, a);
    const int batch = (int)(nw / G.m[a]);
    cufftHandle p = 0;
    if (cufftPlanMany(&p, 1, &L, nullptr, 1, L, nullptr, 1, L, CUFFT_Z2Z, batch) != CUFFT_SUCCESS)
      return set_error(ctx, EMSESG_ERR_CUDA, "cufftPlanMany (Z2Z, %d x %d) failed", L, batch);
    s.gplan[a] = (int)p;
    s.has_gplan[a] = true;
    if (cufftSetStream(p, ctx->stream) != CUFFT_SUCCESS) return set_error(ctx, EMSESG_ERR_CUDA, "cufftSetStream failed");
  }
  for (int a = 0; a < 3; a++) s.gt[a] = t[a];
  return EMSESG_OK;
}

// One axis's r2r transform of every line of w (kind as k_es_line_in).
int es_axis(emsesg_ctx* ctx, const EsGeo& G, int a, int kind) {
  EsState& s = ctx->es;
  const int L = es_line_len(G, a);
  const int64_t lines = (int64_t)G.m[0] * G.m[1] * G.m[2] / G.m[a];
  cufftDoubleComplex* z = static_cast<cufftDoubleComplex*>(s.z);
  EMSESG_LAUNCH(ctx, "es_lines", k_es_line_in, es_blocks(lines * L), ES_BLOCK, 0, s.w, G, a, kind, L, lines, z);
  timer_begin(ctx, "es_fft");
  const cufftResult r = cufftExecZ2Z((cufftHandle)s.gplan[a], z, z, kind == 1 ? CUFFT_INVERSE : CUFFT_FORWARD);
  timer_end(ctx);
  if (r != CUFFT_SUCCESS) return set_error(ctx, EMSESG_ERR_CUDA, "cufftExecZ2Z failed (%d)", (int)r);
  EMSESG_LAUNCH(ctx, "es_lines", k_es_line_out, es_blocks(lines * G.m[a]), ES_BLOCK, 0, z, G, a, kind, L, lines,
                s.w);
  return EMSESG_OK;
}

// phi for any field boundary: pack (with the Neumann values), forward along
// x, y, then z, divide, back along z, then x and y, unpack with the guards.
int es_solve_general(emsesg_ctx* ctx, const int* t, const EsBc& bc) {
  int rc = es_setup_general(ctx, t);
  if (rc) return rc;
  EsState& s = ctx->es;
  const emsesg_config& c = ctx->cfg;
  const EsGeo G = es_geo(c, t);
  const int64_t nw = (int64_t)G.m[0] * G.m[1] * G.m[2];
  const FieldDesc fr = field_desc(c, EMSESG_FIELD_RHO), fp = field_desc(c, EMSESG_FIELD_PHI);
  EMSESG_LAUNCH(ctx, "es_pack", k_es_pack_w, es_blocks(nw), ES_BLOCK, 0, ctx->field[EMSESG_FIELD_RHO], fr, G, bc,
                s.w);
  const int fwd[3] = {t[0] == 0 ? 0 : t[0] + 1, t[1] == 0 ? 0 : t[1] + 1, t[2] == 0 ? 0 : t[2] + 1};
  const int inv[3] = {t[0] == 0 ? 1 : t[0] + 1, t[1] == 0 ? 1 : t[1] + 1, t[2] == 0 ? 1 : t[2] + 1};
  for (int a : {0, 1, 2})
    if ((rc = es_axis(ctx, G, a, fwd[a]))) return rc;
  double mfactor = 1.0;
  for (int a = 0; a < 3; a++) mfactor *= t[a] == 0 ? (double)G.n[a] : 2.0 * G.n[a];
  EMSESG_LAUNCH(ctx, "es_divide", k_es_divide_w, es_blocks(nw), ES_BLOCK, 0, s.w, s.glam, s.glam + G.m[0],
                s.glam + G.m[0] + G.m[1], G, mfactor);
  for (int a : {2, 0, 1})
    if ((rc = es_axis(ctx, G, a, inv[a]))) return rc;
  EMSESG_LAUNCH(ctx, "es_unpack", k_es_unpack_w, es_blocks(fp.size()), ES_BLOCK, 0, s.w,
                ctx->field[EMSESG_FIELD_PHI], fp, G);
  return EMSESG_OK;
}

}  // namespace

void es_free(emsesg_ctx* ctx) {
  EsState& s = ctx->es;
  if (s.has_fwd) cufftDestroy((cufftHandle)s.fwd);
  if (s.has_inv) cufftDestroy((cufftHandle)s.inv);
  es_free_general(s);
  cudaFree(s.r);
  cudaFree(s.c);
  cudaFree(s.lam);
  cudaFree(s.sum);
  s = EsState{};
}

}  // namespace emsesg

using namespace emsesg;

extern "C" int emsesg_esfield(emsesg_ctx* ctx, const int* mtd_vbnd, const double* bcond, int mltstp,
                              double* resid) {
  if (!ctx || mltstp < 1) return EMSESG_ERR_ARG;
  const emsesg_config& c = ctx->cfg;
  int t[3] = {0, 0, 0};
  const int n3[3] = {c.nx, c.ny, c.nz};
  for (int d = 0; d < 3; d++) {
    t[d] = mtd_vbnd ? mtd_vbnd[d] : 0;
    if (t[d] < 0 || t[d] > 2) return set_error(ctx, EMSESG_ERR_ARG, "mtd_vbnd(%d) = %d: 0, 1 or 2", d + 1, t[d]);
    if (t[d] != 0 && n3[d] < 2) return set_error(ctx, EMSESG_ERR_ARG, "a field face needs two cells or more");
  }
  EsBc bc{};
  for (int q = 0; q < 6; q++) bc.v[q] = bcond ? bcond[q] : 0.0;
  int rc = apply_pending_eb(ctx);
  if (rc) return rc;
  const bool periodic = t[0] == 0 && t[1] == 0 && t[2] == 0;
  EsState& s = ctx->es;
  const int nx = c.nx, ny = c.ny, nz = c.nz, nxh = nx / 2 + 1;
  const int64_t n = (int64_t)nx * ny * nz, nh = (int64_t)nxh * ny * nz;
  const FieldDesc fr = field_desc(c, EMSESG_FIELD_RHO), fp = field_desc(c, EMSESG_FIELD_PHI),
                  fe = field_desc(c, EMSESG_FIELD_EB);
  double* rho = ctx->field[EMSESG_FIELD_RHO];
  double* phi = ctx->field[EMSESG_FIELD_PHI];
  if (periodic) {
    if ((rc = es_setup(ctx))) {
      es_free(ctx);  // a partial set-up is made again on the next call
      return rc;
    }
    EMSESG_LAUNCH(ctx, "es_pack", k_es_pack, es_blocks(n), ES_BLOCK, 0, rho, fr, nx, ny, nz, s.r);
    timer_begin(ctx, "es_fft");
    cufftResult fr1 = cufftExecD2Z((cufftHandle)s.fwd, s.r, static_cast<cufftDoubleComplex*>(s.c));
    timer_end(ctx);
    if (fr1 != CUFFT_SUCCESS) return set_error(ctx, EMSESG_ERR_CUDA, "cufftExecD2Z failed (%d)", (int)fr1);
    EMSESG_LAUNCH(ctx, "es_divide", k_es_divide, es_blocks(nh), ES_BLOCK, 0, static_cast<cufftDoubleComplex*>(s.c),
                  s.lam, s.lam + nxh, s.lam + nxh + ny, nxh, ny, nz, (double)n);
    timer_begin(ctx, "es_fft");
    cufftResult fr2 = cufftExecZ2D((cufftHandle)s.inv, static_cast<cufftDoubleComplex*>(s.c), s.r);
    timer_end(ctx);
    if (fr2 != CUFFT_SUCCESS) return set_error(ctx, EMSESG_ERR_CUDA, "cufftExecZ2D failed (%d)", (int)fr2);
    EMSESG_LAUNCH(ctx, "es_unpack", k_es_unpack, es_blocks(fp.size()), ES_BLOCK, 0, s.r, phi, fp, nx, ny, nz);
  } else if ((rc = es_solve_general(ctx, t, bc))) {
    es_free_general(s);
    return rc;
  }
  EMSESG_LAUNCH(ctx, "es_efield", k_es_efield, es_blocks((int64_t)fe.ex * fe.ey * fe.ez), ES_BLOCK, 0, phi, fp,
                ctx->field[EMSESG_FIELD_EB], fe, nx, ny, nz, (double)mltstp, t[0], t[1], t[2]);
  if (resid) {
    // poichk's loop: from the first solved node to min(n - 1, the last)
    const EsGeo G = es_geo(c, t);
    int lo[3], cnt[3];
    for (int d = 0; d < 3; d++) {
      lo[d] = G.lo[d];
      cnt[d] = std::min(G.n[d] - 1, G.lo[d] + G.m[d] - 1) - G.lo[d] + 1;
    }
    const int64_t nc = (int64_t)cnt[0] * cnt[1] * cnt[2];
    if (!s.sum) EMSESG_CUDA(ctx, cudaMalloc(&s.sum, sizeof(double)));
    EMSESG_CUDA(ctx, cudaMemsetAsync(s.sum, 0, sizeof(double), ctx->stream));
    EMSESG_LAUNCH(ctx, "es_poichk", k_es_poichk, es_blocks(nc), ES_BLOCK, 0, rho, fr, phi, fp, lo[0], lo[1], lo[2],
                  cnt[0], cnt[1], cnt[2], s.sum);
    double sum = 0.0;
    EMSESG_CUDA(ctx, cudaMemcpyAsync(&sum, s.sum, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    EMSESG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *resid = std::sqrt(sum) / (double)nc;
  }
  return EMSESG_OK;
}
