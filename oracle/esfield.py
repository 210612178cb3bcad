"""TEST INFRASTRUCTURE ONLY: the FP64 restatement of the reference's
electrostatic field step, the checker of emsesg_esfield.  Only tests/ (and
bench.py's checks) use it.

It follows the reference's own sequence, on a single rank (pftmode 3/4):

* poisson(3), src/field/poisson/poissn.F90:64-470 with the set-up of
  src/field/poisson/inifft.F90:389-470, per axis by its mtd_vbnd:
  0 (periodic) the nodes 0..n-1, FFTW_R2HC / FFTW_HC2R,
  kmod(i) = (2 sin(pi i / n) / dr)^2 in the halfcomplex slot order
  (i = 0..n/2, then (n+1)/2-1 down to 1), mfactor n;
  1 (phi = 0 on the faces) the nodes 1..n-1, FFTW_RODFT00 both ways,
  kmod(i) = 2 (1 - cos(i pi / n)) / dr^2 on node i, mfactor 2n;
  2 (Neumann) the nodes 0..n, FFTW_REDFT00 both ways, the same kmod,
  mfactor 2n, and rho_tilde = rho - 2 bc(1) on the node-0 plane and
  + 2 bc(2) on the node-n plane (poissn.F90:76-127; bc = the reference's
  boundary_conditions(side, axis) * rene);
  forward along x and y, then z; every coefficient divided by
  (kmod_x + kmod_y + kmod_z) * mfactor, a zero divisor giving 0; back along
  z, then x and y.  FFTW's halfcomplex layout (r_0, r_1, ..., r_{n/2},
  i_{(n+1)/2-1}, ..., i_1) is built from numpy's real FFT (same sign
  convention); RODFT00 and REDFT00 are scipy's type-1 DST and DCT, whose
  unnormalised definitions are FFTW's.
* the guards (poissn.F90:672-710): zero outside every axis's solved nodes,
  then the periodic copies phi(-1) = phi(n-1), phi(n) = phi(0),
  phi(n+1) = phi(1) on periodic axes;
* esfld2, src/field/esfild.F90:351-435: EX..EZ = 0, then
  EX(i,j,k) = (phi(i,j,k) - phi(i+1,j,k)) * mltstp on i = -1..n, j, k = 0..n,
  likewise for EY, EZ; on an axis with mtd_vbnd 1 the normal component at
  -1 and n copies the one at 0 and n-1, with mtd_vbnd 2 it takes its
  negative;
* poichk, poissn.F90:921-961: sqrt(sum of (rho + sum of the six
  neighbours of phi - 6 phi)^2 over the solved nodes, a Neumann axis up to
  node n-1) / their count.

Arrays use the numpy layout of ctca_b200.emses.field_shape: (z, y, x, comp)
with index [k+1, j+1, i+1, c] for Fortran field(c+1, i, j, k) (lower guard -1).
"""
from __future__ import annotations

import numpy as np
import scipy.fft as sfft


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


# ---------------------------------------------------------------- any mtd_vbnd

def solve_range(n: int, t: int) -> tuple[int, int]:
    """First and last solved node of an axis of n cells with mtd_vbnd t."""
    return {0: (0, n - 1), 1: (1, n - 1), 2: (0, n)}[t]


def kmod_axis(n: int, t: int, dr: float = 1.0) -> np.ndarray:
    """kmod(:, :, 2) over an axis's solved nodes (or halfcomplex slots)."""
    if t == 0:
        return kmod(n, dr)
    lo, hi = solve_range(n, t)
    pi, dri = np.arccos(-1.0), 1.0 / dr
    return np.array([2.0 * (1.0 - np.cos(i * pi / n)) * dri * dri for i in range(lo, hi + 1)])


def _fwd(a, axis, t):
    if t == 0:
        return r2hc(a, axis)
    return sfft.dst(a, type=1, axis=axis) if t == 1 else sfft.dct(a, type=1, axis=axis)


def _inv(a, axis, t):
    if t == 0:
        return hc2r(a, axis)
    return sfft.dst(a, type=1, axis=axis) if t == 1 else sfft.dct(a, type=1, axis=axis)


def poisson_general(rho_f: np.ndarray, mtd, bc=None) -> np.ndarray:
    """phi field (nodes -1..n+1, guards as the reference sets them) from the
    rho field for mtd_vbnd = mtd (x, y, z) and the Neumann values bc[axis][side]
    (boundary_conditions(side, axis) * rene)."""
    nz, ny, nx = (s - 3 for s in rho_f.shape[:3])
    n = (nx, ny, nz)
    rt = np.array(rho_f[..., 0], dtype=np.float64)   # rho_tilde, [k+1, j+1, i+1]
    for d in range(3):                                # x, y, z
        if mtd[d] == 2:
            b = bc[d] if bc is not None else (0.0, 0.0)
            ax = 2 - d
            lo = [slice(None)] * 3
            hi = [slice(None)] * 3
            lo[ax] = 1          # node 0
            hi[ax] = n[d] + 1   # node n
            rt[tuple(lo)] = rt[tuple(lo)] - b[0] * 2.0
            rt[tuple(hi)] = rt[tuple(hi)] + b[1] * 2.0
    rng = [solve_range(n[d], mtd[d]) for d in range(3)]
    sl = tuple(slice(rng[d][0] + 1, rng[d][1] + 2) for d in (2, 1, 0))
    poi = rt[sl]
    poi = _fwd(_fwd(poi, 2, mtd[0]), 1, mtd[1])       # FFT-xy
    poi = _fwd(poi, 0, mtd[2])                        # FFT-z
    mf = 1.0
    for d in range(3):
        mf *= n[d] if mtd[d] == 0 else 2.0 * n[d]
    div = (kmod_axis(nx, mtd[0])[None, None, :] + kmod_axis(ny, mtd[1])[None, :, None]
           + kmod_axis(nz, mtd[2])[:, None, None]) * mf
    with np.errstate(divide="ignore", invalid="ignore"):
        poi = np.where(div != 0.0, poi / np.where(div != 0.0, div, 1.0), 0.0)
    poi = _inv(poi, 0, mtd[2])
    poi = _inv(_inv(poi, 2, mtd[0]), 1, mtd[1])
    phi = np.zeros_like(rt)
    phi[sl] = poi
    for d in range(3):                                # periodic copies
        if mtd[d] == 0:
            ax = 2 - d
            def cp(dst, src):
                a = [slice(None)] * 3
                b = [slice(None)] * 3
                a[ax] = dst + 1
                b[ax] = src + 1
                phi[tuple(a)] = phi[tuple(b)]
            cp(-1, n[d] - 1)
            cp(n[d], 0)
            cp(n[d] + 1, 1)
    return phi[..., None]


def esfield_general(rho_f, eb_f, mtd, bc=None, mltstp: int = 1):
    """(phi field, eb field) of emsesg_esfield for any mtd_vbnd."""
    nz, ny, nx = (s - 3 for s in rho_f.shape[:3])
    n = (nx, ny, nz)
    phi = poisson_general(rho_f, mtd, bc)
    eb = np.array(eb_f, dtype=np.float64)
    eb[..., 0:3] = 0.0
    p = phi[..., 0]
    m = float(mltstp)
    eb[1:nz + 2, 1:ny + 2, 0:nx + 2, 0] = (p[1:nz + 2, 1:ny + 2, 0:nx + 2] - p[1:nz + 2, 1:ny + 2, 1:nx + 3]) * m
    eb[1:nz + 2, 0:ny + 2, 1:nx + 2, 1] = (p[1:nz + 2, 0:ny + 2, 1:nx + 2] - p[1:nz + 2, 1:ny + 3, 1:nx + 2]) * m
    eb[0:nz + 2, 1:ny + 2, 1:nx + 2, 2] = (p[0:nz + 2, 1:ny + 2, 1:nx + 2] - p[1:nz + 3, 1:ny + 2, 1:nx + 2]) * m
    for d in range(3):
        if mtd[d] == 0:
            continue
        sgn = 1.0 if mtd[d] == 1 else -1.0
        ax = 2 - d
        other = [slice(1, n[e] + 2) for e in (2, 1, 0)]   # nodes 0..n of the other axes
        def at(node):
            idx = list(other)
            idx[ax] = node + 1
            return tuple(idx) + (d,)
        eb[at(-1)] = sgn * eb[at(0)]
        eb[at(n[d])] = sgn * eb[at(n[d] - 1)]
    return phi, eb


def poichk_general(rho_f, phi_f, mtd) -> float:
    """poichk's residual over the nodes lfft..min(n-1, ufft) of every axis
    (its loop bounds, poissn.F90:937-939: a Neumann axis stops at n-1)."""
    nz, ny, nx = (s - 3 for s in rho_f.shape[:3])
    n = (nx, ny, nz)
    rng = [(solve_range(n[d], mtd[d])[0], min(n[d] - 1, solve_range(n[d], mtd[d])[1])) for d in range(3)]
    p = phi_f[..., 0]
    r = rho_f[..., 0]
    tot, cnt = 0.0, 0
    (x0, x1), (y0, y1), (z0, z1) = rng
    c = (slice(z0 + 1, z1 + 2), slice(y0 + 1, y1 + 2), slice(x0 + 1, x1 + 2))
    def sh(dz, dy, dx):
        return p[z0 + 1 + dz:z1 + 2 + dz, y0 + 1 + dy:y1 + 2 + dy, x0 + 1 + dx:x1 + 2 + dx]
    d = r[c] + (sh(0, 0, -1) + sh(0, 0, 1) + sh(0, -1, 0) + sh(0, 1, 0) + sh(-1, 0, 0) + sh(1, 0, 0)) - 6.0 * p[c]
    return float(np.sqrt(np.sum(d * d)) / d.size)
