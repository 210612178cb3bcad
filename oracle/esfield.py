"""TEST INFRASTRUCTURE ONLY: the FP64 restatement of the reference's
electrostatic field step for periodic fields, the checker of
emsesg_esfield.  Only tests/ (and bench.py's checks) use it.

It follows the reference's own sequence:

* poisson(3), src/field/poisson/poissn.F90:216-470 with the periodic set-up
  of src/field/poisson/inifft.F90:389-470: rho on the nodes 0..n-1 of every
  axis goes through FFTW's real-to-halfcomplex transform (FFTW_R2HC,
  unnormalised) along x and y, then z; every halfcomplex coefficient (i, j, k)
  is divided by (kmod_x(i) + kmod_y(j) + kmod_z(k)) * mfactor, with
  kmod(m) = (2 sin(pi i / n) / dr)^2 in the halfcomplex order of the slots
  (i = 0..n/2, then (n+1)/2-1 down to 1) and mfactor = nx ny nz; a zero
  divisor (the mean) gives 0; then FFTW_HC2R along z, then x and y.  FFTW's
  halfcomplex layout (r_0, r_1, ..., r_{n/2}, i_{(n+1)/2-1}, ..., i_1) is
  built here from numpy's real FFT, which has the same sign convention.
* the periodic guards of poissn.F90:686-710: phi(-1) = phi(n-1),
  phi(n) = phi(0), phi(n+1) = phi(1) on every axis;
* esfld2, src/field/esfild.F90:351-366: EX..EZ = 0, then
  EX(i,j,k) = (phi(i,j,k) - phi(i+1,j,k)) * mltstp on i = -1..n, j, k = 0..n,
  likewise for EY, EZ;
* poichk, poissn.F90:921-961: sqrt(sum of (rho + sum of the six
  neighbours of phi - 6 phi)^2 over the nodes 0..n-1) / their count.

Arrays use the numpy layout of ctca_b200.emses.field_shape: (z, y, x, comp)
with index [k+1, j+1, i+1, c] for Fortran field(c+1, i, j, k) (lower guard -1).
"""
from __future__ import annotations

import numpy as np


def r2hc(x: np.ndarray, axis: int) -> np.ndarray:
    """FFTW_R2HC along one axis (unnormalised)."""
    n = x.shape[axis]
    X = np.fft.rfft(x, axis=axis)
    re = np.take(X.real, np.arange(0, n // 2 + 1), axis=axis)
    im = np.take(X.imag, np.arange((n + 1) // 2 - 1, 0, -1), axis=axis)
    return np.concatenate([re, im], axis=axis)


def hc2r(h: np.ndarray, axis: int) -> np.ndarray:
    """FFTW_HC2R along one axis (unnormalised: hc2r(r2hc(x)) = n x)."""
    n = h.shape[axis]
    re = np.take(h, np.arange(0, n // 2 + 1), axis=axis)
    im = np.zeros_like(re)
    nim = (n + 1) // 2 - 1  # imaginary parts i_1 .. i_nim, stored in reverse
    if nim > 0:
        tail = np.take(h, np.arange(n // 2 + 1, n), axis=axis)  # i_nim .. i_1
        sl = [slice(None)] * h.ndim
        sl[axis] = slice(1, nim + 1)
        im[tuple(sl)] = np.flip(tail, axis=axis)
    return np.fft.irfft(re + 1j * im, n=n, axis=axis) * n


def kmod(n: int, dr: float = 1.0) -> np.ndarray:
    """kmod(:, :, 2) of a periodic axis in the halfcomplex slot order
    (inifft.F90:392-403)."""
    pi, rn, dri = np.arccos(-1.0), 1.0 / n, 1.0 / dr
    out = []
    for i in list(range(0, n // 2 + 1)) + list(range((n + 1) // 2 - 1, 0, -1)):
        k = 2.0 * np.sin(pi * i * rn) * dri
        out.append(k * k)
    return np.array(out)


def poisson_nodes(rho: np.ndarray) -> np.ndarray:
    """phi on the nodes 0..n-1 (array (nz, ny, nx)) from rho on the same
    nodes, by the reference's transforms and division."""
    nz, ny, nx = rho.shape
    poi = np.array(rho, dtype=np.float64)
    poi = r2hc(r2hc(poi, 2), 1)          # FFT-xy
    poi = r2hc(poi, 0)                   # FFT-z
    div = (kmod(nx)[None, None, :] + kmod(ny)[None, :, None] + kmod(nz)[:, None, None]) * float(nx * ny * nz)
    with np.errstate(divide="ignore", invalid="ignore"):
        poi = np.where(div != 0.0, poi / np.where(div != 0.0, div, 1.0), 0.0)
    poi = hc2r(poi, 0)                   # inverse FFT-z
    return hc2r(hc2r(poi, 2), 1)         # inverse FFT-xy


def phi_field(phin: np.ndarray) -> np.ndarray:
    """phi on the nodes -1..n+1 with the periodic guards, field layout."""
    nz, ny, nx = phin.shape
    idx = lambda n: (np.arange(-1, n + 2) + n) % n
    p = phin[np.ix_(idx(nz), idx(ny), idx(nx))]
    return p[..., None]


def esfield(rho_f: np.ndarray, eb_f: np.ndarray, mltstp: int = 1):
    """(phi field, eb field) of emsesg_esfield from the rho field and eb
    (BX..BZ kept).  Fields in the numpy layout described above."""
    nz, ny, nx = (s - 3 for s in rho_f.shape[:3])
    rho = rho_f[1:nz + 1, 1:ny + 1, 1:nx + 1, 0]   # nodes 0..n-1
    phi = phi_field(poisson_nodes(rho))
    eb = np.array(eb_f, dtype=np.float64)
    eb[..., 0:3] = 0.0
    p = phi[..., 0]
    m = float(mltstp)
    # EX on i = -1..n (array x index 0..n+1), j, k = 0..n
    eb[1:nz + 2, 1:ny + 2, 0:nx + 2, 0] = (p[1:nz + 2, 1:ny + 2, 0:nx + 2] - p[1:nz + 2, 1:ny + 2, 1:nx + 3]) * m
    eb[1:nz + 2, 0:ny + 2, 1:nx + 2, 1] = (p[1:nz + 2, 0:ny + 2, 1:nx + 2] - p[1:nz + 2, 1:ny + 3, 1:nx + 2]) * m
    eb[0:nz + 2, 1:ny + 2, 1:nx + 2, 2] = (p[0:nz + 2, 1:ny + 2, 1:nx + 2] - p[1:nz + 3, 1:ny + 2, 1:nx + 2]) * m
    return phi, eb


def poichk(rho_f: np.ndarray, phi_f: np.ndarray) -> float:
    """poichk's residual over the nodes 0..n-1."""
    nz, ny, nx = (s - 3 for s in rho_f.shape[:3])
    r = rho_f[1:nz + 1, 1:ny + 1, 1:nx + 1, 0]
    p = phi_f[..., 0]
    c = p[1:nz + 1, 1:ny + 1, 1:nx + 1]
    nb = (p[1:nz + 1, 1:ny + 1, 0:nx] + p[1:nz + 1, 1:ny + 1, 2:nx + 2] + p[1:nz + 1, 0:ny, 1:nx + 1]
          + p[1:nz + 1, 2:ny + 2, 1:nx + 1] + p[0:nz, 1:ny + 1, 1:nx + 1] + p[2:nz + 2, 1:ny + 1, 1:nx + 1])
    d = r + nb - 6.0 * c
    return float(np.sqrt(np.sum(d * d)) / d.size)
