"""The oracle of the electrostatic field step (oracle/esfield.py) against
what the reference's algorithm must give, without a GPU:

* FFTW's halfcomplex transforms as restated: hc2r(r2hc(x)) = n x, and r2hc
  of a cosine / sine puts n/2 in the slot of its frequency (real part in
  slot k, imaginary part in slot n - k);
* a single Fourier mode of rho gives phi = rho / lambda with lambda the
  7-point Laplacian's eigenvalue sum_d (2 sin(pi k_d / n_d))^2: the division
  by kmod in the halfcomplex slot order is the right one for every slot;
* for any rho the result satisfies the reference's own check (poichk's
  stencil, poissn.F90:937-943): rho + sum of the six neighbours - 6 phi =
  mean(rho) on every node, with mean(phi) = 0;
* esfld2's staggered differences and the periodic guards."""
import numpy as np
import pytest

from oracle import esfield as E


@pytest.mark.parametrize("n", [8, 9, 16, 15])
def test_halfcomplex_transforms(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal((3, n))
    assert np.allclose(E.hc2r(E.r2hc(x, 1), 1), n * x, rtol=0, atol=1e-12 * n)
    j = np.arange(n)
    for k in range(1, (n + 1) // 2):
        h = E.r2hc(np.cos(2 * np.pi * k * j / n)[None, :], 1)[0]
        want = np.zeros(n)
        want[k] = n / 2
        assert np.allclose(h, want, atol=1e-12 * n), k
        h = E.r2hc(np.sin(2 * np.pi * k * j / n)[None, :], 1)[0]
        want = np.zeros(n)
        want[n - k] = -n / 2  # FFTW's sign: X_k = sum x_j exp(-2 pi i j k / n)
        assert np.allclose(h, want, atol=1e-12 * n), k


def rho_field(rho_nodes):
    """Nodes 0..n-1 -> the rho field (nodes -1..n+1, periodic)."""
    return E.phi_field(rho_nodes)


@pytest.mark.parametrize("shape,mode", [((8, 8, 8), (1, 2, 3)), ((12, 10, 16), (5, 0, 7)),
                                        ((9, 15, 14), (4, 7, 1)), ((16, 16, 16), (8, 8, 8))])
def test_single_mode_is_divided_by_its_eigenvalue(shape, mode):
    nz, ny, nx = shape
    c, b, a = mode
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    arg = 2 * np.pi * (a * i / nx + b * j / ny + c * k / nz)
    lam = sum((2 * np.sin(np.pi * m / n)) ** 2 for m, n in ((a, nx), (b, ny), (c, nz)))
    for f in (np.cos, np.sin):
        rho = f(arg) + 0.3 * np.cos(arg + 0.7)
        phi = E.poisson_nodes(rho)
        assert np.allclose(phi, rho / lam, rtol=0, atol=1e-12 * np.abs(rho).max() / lam)


@pytest.mark.parametrize("shape", [(8, 8, 8), (10, 12, 14), (9, 7, 11)])
def test_solution_satisfies_the_reference_check(shape):
    rng = np.random.default_rng(sum(shape))
    rho = rng.standard_normal(shape)
    phi = E.poisson_nodes(rho)
    assert abs(phi.mean()) < 1e-14 * np.abs(phi).max()
    pf = E.phi_field(phi)
    # zero-mean rho: poichk's residual vanishes to rounding
    r0 = rho - rho.mean()
    p0 = E.phi_field(E.poisson_nodes(r0))
    assert E.poichk(rho_field(r0), p0) < 1e-14 * np.abs(r0).max()
    # else every node keeps mean(rho): residual = |mean| / sqrt(N)
    assert np.isclose(E.poichk(rho_field(rho), pf), abs(rho.mean()) / np.sqrt(rho.size), rtol=1e-9)


def test_esfld2_differences_and_guards():
    rng = np.random.default_rng(5)
    nz, ny, nx = 6, 7, 8
    rho = rng.standard_normal((nz, ny, nx))
    rho -= rho.mean()
    eb0 = rng.standard_normal((nz + 3, ny + 3, nx + 3, 6))
    phi, eb = E.esfield(rho_field(rho), eb0, mltstp=3)
    p = phi[..., 0]
    # periodic guards
    assert np.array_equal(p[0], p[nz]) and np.array_equal(p[nz + 1], p[1]) and np.array_equal(p[nz + 2], p[2])
    assert np.array_equal(p[:, :, 0], p[:, :, nx]) and np.array_equal(p[:, :, nx + 2], p[:, :, 2])
    # B untouched
    assert np.array_equal(eb[..., 3:], eb0[..., 3:])
    # EX(i, j, k) = 3 (phi(i) - phi(i+1)) for i = -1..n, j, k = 0..n; zero elsewhere
    for (k, j, i) in [(0, 0, -1), (3, 5, 2), (nz, ny, nx), (2, 0, nx)]:
        assert eb[k + 1, j + 1, i + 1, 0] == 3.0 * (p[k + 1, j + 1, i + 1] - p[k + 1, j + 1, i + 2])
    assert np.all(eb[:, 0, :, 0] == 0) and np.all(eb[:, :, nx + 2, 0] == 0) and np.all(eb[0, :, :, 0] == 0)
    assert np.all(eb[:, :, 0, 1] == 0) and np.all(eb[:, ny + 2, :, 1] == 0)
    assert np.all(eb[nz + 2, :, :, 2] == 0) and np.all(eb[:, 0, :, 2] == 0)
    # the discrete divergence of E is rho (times mltstp) on the nodes 0..n-1
    ex, ey, ez = eb[..., 0], eb[..., 1], eb[..., 2]
    div = ((ex[1:nz + 1, 1:ny + 1, 1:nx + 1] - ex[1:nz + 1, 1:ny + 1, 0:nx])
           + (ey[1:nz + 1, 1:ny + 1, 1:nx + 1] - ey[1:nz + 1, 0:ny, 1:nx + 1])
           + (ez[1:nz + 1, 1:ny + 1, 1:nx + 1] - ez[0:nz, 1:ny + 1, 1:nx + 1]))
    assert np.allclose(div, 3.0 * rho, atol=1e-12 * np.abs(rho).max())
