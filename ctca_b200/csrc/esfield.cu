// esfield.cu -- the electrostatic field step of the reference on the device,
// for periodic fields: esfld1(0) with poisson(3) (the FFT solution of the
// discrete Poisson equation), the periodic guards of phi, esfld2 (E on its
// staggered positions from phi) and poichk (the residual of the discrete
// equation).  FP64 throughout, like the reference's field arrays.
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
// the transforms.
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
                            int nx, int ny, int nz, double mlt) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)fe.ex * fe.ey * fe.ez) return;
  const int i = (int)(t % fe.ex) + fe.lo, j = (int)((t / fe.ex) % fe.ey) + fe.lo,
            k = (int)(t / ((int64_t)fe.ex * fe.ey)) + fe.lo;
  const bool jk = j >= 0 && j <= ny && k >= 0 && k <= nz;
  const bool ik = i >= 0 && i <= nx && k >= 0 && k <= nz;
  const bool ij = i >= 0 && i <= nx && j >= 0 && j <= ny;
  const double p = (i <= nx + 1 && j <= ny + 1 && k <= nz + 1) ? phi[fp.at(0, i, j, k)] : 0.0;
  eb[fe.at(0, i, j, k)] = (jk && i <= nx) ? (p - phi[fp.at(0, i + 1, j, k)]) * mlt : 0.0;
  eb[fe.at(1, i, j, k)] = (ik && j <= ny) ? (p - phi[fp.at(0, i, j + 1, k)]) * mlt : 0.0;
  eb[fe.at(2, i, j, k)] = (ij && k <= nz) ? (p - phi[fp.at(0, i, j, k + 1)]) * mlt : 0.0;
}

// poichk (poissn.F90:937-948): the sum of squares of
// rho + (phi(i-1) + phi(i+1) + phi(j-1) + phi(j+1) + phi(k-1) + phi(k+1)) - 6 phi
// over the nodes 0..n-1, in the order of the terms there; one atomic per block.
__global__ void k_es_poichk(const double* __restrict__ rho, FieldDesc fr, const double* __restrict__ phi,
                            FieldDesc fp, int nx, int ny, int nz, double* __restrict__ sum) {
  __shared__ double part[ES_BLOCK / 32];
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double d2 = 0.0;
  if (t < (int64_t)nx * ny * nz) {
    const int i = (int)(t % nx), j = (int)((t / nx) % ny), k = (int)(t / ((int64_t)nx * ny));
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
  EMSESG_CUDA(ctx, cudaMalloc(&s.sum, sizeof(double)));
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

}  // namespace

void es_free(emsesg_ctx* ctx) {
  EsState& s = ctx->es;
  if (s.has_fwd) cufftDestroy((cufftHandle)s.fwd);
  if (s.has_inv) cufftDestroy((cufftHandle)s.inv);
  cudaFree(s.r);
  cudaFree(s.c);
  cudaFree(s.lam);
  cudaFree(s.sum);
  s = EsState{};
}

}  // namespace emsesg

using namespace emsesg;

extern "C" int emsesg_esfield(emsesg_ctx* ctx, int mltstp, double* resid) {
  if (!ctx || mltstp < 1) return EMSESG_ERR_ARG;
  const emsesg_config& c = ctx->cfg;
  for (int d = 0; d < 3; d++)
    if (c.nfbnd[d] != 0)
      return set_error(ctx, EMSESG_ERR_UNSUPPORTED, "electrostatic field: periodic fields only (mtd_vbnd = 0)");
  int rc = apply_pending_eb(ctx);
  if (rc) return rc;
  if ((rc = es_setup(ctx))) {
    es_free(ctx);  // a partial set-up is made again on the next call
    return rc;
  }
  EsState& s = ctx->es;
  const int nx = c.nx, ny = c.ny, nz = c.nz, nxh = nx / 2 + 1;
  const int64_t n = (int64_t)nx * ny * nz, nh = (int64_t)nxh * ny * nz;
  const FieldDesc fr = field_desc(c, EMSESG_FIELD_RHO), fp = field_desc(c, EMSESG_FIELD_PHI),
                  fe = field_desc(c, EMSESG_FIELD_EB);
  double* rho = ctx->field[EMSESG_FIELD_RHO];
  double* phi = ctx->field[EMSESG_FIELD_PHI];
  EMSESG_LAUNCH(ctx, "es_pack", k_es_pack, es_blocks(n), ES_BLOCK, 0, rho, fr, nx, ny, nz, s.r);
  timer_begin(ctx, "es_fft");
  cufftResult fr1 = cufftExecD2Z((cufftHandle)s.fwd, s.r, static_cast<cufftDoubleComplex*>(s.c));
  timer_end(ctx);
  if (fr1 != CUFFT_SUCCESS) return set_error(ctx, EMSESG_ERR_CUDA, "cufftExecD2Z failed (%d)", (int)fr1);
  EMSESG_LAUNCH(ctx, "es_divide", k_es_divide, es_blocks(nh), ES_BLOCK, 0, static_cast<cufftDoubleComplex*>(s.c), s.lam, s.lam + nxh,
                s.lam + nxh + ny, nxh, ny, nz, (double)n);
  timer_begin(ctx, "es_fft");
  cufftResult fr2 = cufftExecZ2D((cufftHandle)s.inv, static_cast<cufftDoubleComplex*>(s.c), s.r);
  timer_end(ctx);
  if (fr2 != CUFFT_SUCCESS) return set_error(ctx, EMSESG_ERR_CUDA, "cufftExecZ2D failed (%d)", (int)fr2);
  EMSESG_LAUNCH(ctx, "es_unpack", k_es_unpack, es_blocks(fp.size()), ES_BLOCK, 0, s.r, phi, fp, nx, ny, nz);
  EMSESG_LAUNCH(ctx, "es_efield", k_es_efield, es_blocks((int64_t)fe.ex * fe.ey * fe.ez), ES_BLOCK, 0, phi, fp,
                ctx->field[EMSESG_FIELD_EB], fe, nx, ny, nz, (double)mltstp);
  if (resid) {
    EMSESG_CUDA(ctx, cudaMemsetAsync(s.sum, 0, sizeof(double), ctx->stream));
    EMSESG_LAUNCH(ctx, "es_poichk", k_es_poichk, es_blocks(n), ES_BLOCK, 0, rho, fr, phi, fp, nx, ny, nz, s.sum);
    double sum = 0.0;
    EMSESG_CUDA(ctx, cudaMemcpyAsync(&sum, s.sum, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    EMSESG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *resid = std::sqrt(sum) / (double)n;
  }
  return EMSESG_OK;
}
