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
* esfld2's staggered differences and the periodic guards;
* the other field boundaries (mtd_vbnd 1: phi = 0 on the faces, DST-I;
  2: Neumann, DCT-I): one eigenfunction per axis divided by its eigenvalue,
  the Dirichlet solution exact under poichk's stencil, the Neumann boundary
  values added as the reference adds them, and esfld2's boundary copies."""
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


# ---- other field boundaries (mtd_vbnd 1: phi = 0 on the faces, 2: Neumann)

def nodes_grid(nz, ny, nx):
    return np.meshgrid(np.arange(-1, nz + 2), np.arange(-1, ny + 2), np.arange(-1, nx + 2), indexing="ij")


@pytest.mark.parametrize("mtd,shape,mode", [((1, 0, 0), (8, 9, 10), (3, 2, 1)), ((0, 1, 2), (10, 8, 9), (2, 3, 4)),
                                            ((1, 1, 1), (8, 8, 8), (1, 5, 7)), ((2, 2, 0), (9, 10, 8), (2, 0, 3))])
def test_eigenmodes_of_each_boundary(mtd, shape, mode):
    """A product of one eigenfunction per axis -- cos / sin of 2 pi a i / n
    (periodic), sin(pi a i / n) (phi = 0), cos(pi a i / n) (Neumann) -- is
    divided by its eigenvalue sum_d lambda_d, lambda = (2 sin(pi a / n))^2
    periodic and 2 (1 - cos(pi a / n)) otherwise."""
    nz, ny, nx = shape
    k, j, i = nodes_grid(nz, ny, nx)
    n = (nx, ny, nz)
    idx = (i, j, k)
    f, lam = np.ones_like(i, dtype=float), 0.0
    for d in range(3):
        a = mode[d]
        if mtd[d] == 0:
            f = f * np.cos(2 * np.pi * a * idx[d] / n[d])
            lam += (2 * np.sin(np.pi * a / n[d])) ** 2
        elif mtd[d] == 1:
            f = f * np.sin(np.pi * a * idx[d] / n[d])
            lam += 2 * (1 - np.cos(np.pi * a / n[d]))
        else:
            f = f * np.cos(np.pi * a * idx[d] / n[d])
            lam += 2 * (1 - np.cos(np.pi * a / n[d]))
    rho = f[..., None]
    phi = E.poisson_general(rho, mtd)
    rng = [E.solve_range(n[d], mtd[d]) for d in range(3)]
    sl = tuple(slice(rng[d][0] + 1, rng[d][1] + 2) for d in (2, 1, 0))
    assert np.allclose(phi[sl][..., 0], f[sl] / lam, rtol=0, atol=1e-12 / lam)


def test_dirichlet_solution_satisfies_the_reference_check():
    """phi = 0 on the faces: the solved interior satisfies poichk's stencil
    exactly (no mean to remove), with phi on the faces and guards zero."""
    rng = np.random.default_rng(3)
    nz, ny, nx = 9, 8, 10
    rho = rng.standard_normal((nz + 3, ny + 3, nx + 3, 1))
    phi = E.poisson_general(rho, (1, 1, 1))
    assert E.poichk_general(rho, phi, (1, 1, 1)) < 1e-14 * np.abs(rho).max()
    p = phi[..., 0]
    for face in (p[0], p[1], p[nz + 1], p[nz + 2], p[:, 1], p[:, :, nx + 1]):
        assert np.all(face == 0.0)


def test_neumann_boundary_values_enter_as_the_reference_adds_them():
    """mtd_vbnd 2 with boundary values: the same as the solve of rho_tilde
    (rho - 2 bc(1) on the node-0 plane, + 2 bc(2) on the node-n plane,
    poissn.F90:76-127) without them; guards outside the solved nodes zero."""
    rng = np.random.default_rng(4)
    nz, ny, nx = 8, 9, 10
    rho = rng.standard_normal((nz + 3, ny + 3, nx + 3, 1))
    bc = [(0.0, 0.0), (0.0, 0.0), (0.3, -0.7)]
    a = E.poisson_general(rho, (0, 0, 2), bc)
    rt = rho.copy()
    rt[1] -= 2 * 0.3
    rt[nz + 1] += 2 * -0.7
    b = E.poisson_general(rt, (0, 0, 2))
    assert np.array_equal(a, b)
    assert np.all(a[0] == 0.0) and np.all(a[nz + 2] == 0.0)


@pytest.mark.parametrize("mtd", [(1, 2, 0), (2, 1, 1)])
def test_esfld2_boundary_components(mtd):
    """The normal E component at -1 and n: a copy of the one at 0 and n-1
    with mtd_vbnd 1, its negative with 2 (esfild.F90:368-435)."""
    rng = np.random.default_rng(6)
    nz, ny, nx = 7, 8, 9
    n = (nx, ny, nz)
    rho = rng.standard_normal((nz + 3, ny + 3, nx + 3, 1))
    eb0 = rng.standard_normal((nz + 3, ny + 3, nx + 3, 6))
    phi, eb = E.esfield_general(rho, eb0, mtd, mltstp=2)
    assert np.array_equal(eb[..., 3:], eb0[..., 3:])
    for d in range(3):
        if mtd[d] == 0:
            continue
        s = 1.0 if mtd[d] == 1 else -1.0
        comp = np.moveaxis(eb[..., d], 2 - d, 0)   # the axis first
        inner = tuple(slice(1, n[e] + 2) for e in (2, 1, 0) if e != d)
        assert np.array_equal(comp[(0,) + inner], s * comp[(1,) + inner])
        assert np.array_equal(comp[(n[d] + 1,) + inner], s * comp[(n[d],) + inner])
