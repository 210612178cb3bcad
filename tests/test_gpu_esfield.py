"""emsesg_esfield (the electrostatic field step) against the
oracle's restatement of poisson(3) + esfld2 (oracle/esfield.py), through the
C ABI.

phi and EX..EZ agree with the oracle to 1e-12 relative (the two FFTs round
differently; the eigenvalues are the same doubles), BX..BZ are left
bit-identical, the guards of phi are the periodic copies, and poichk's
residual is at rounding level for a zero-mean rho and |mean| / sqrt(N)
otherwise -- on cubic grids, even and odd sizes, and with mltstp > 1; the
same against the oracle's general solve for every mix of field boundaries
(phi = 0 faces by a type-1 DST, Neumann faces with boundary values by a
type-1 DCT, periodic axes by the halfcomplex transform).  Then
the field goes into the FP32 push: an ES loop (fx_step, esfield, fx_step)
runs and keeps the discrete Gauss law div E = rho - mean(rho)."""
import numpy as np
import pytest

from ctca_b200.emses import Emses, field_shape
from oracle import esfield as E

from helpers import build, case, rel_l2

pytestmark = pytest.mark.gpu


def rho_of(cfg, rng, mean=0.0):
    nodes = rng.standard_normal((cfg.nz, cfg.ny, cfg.nx))
    nodes = nodes - nodes.mean() + mean
    return E.phi_field(nodes)  # nodes -1..n+1, periodic


@pytest.mark.parametrize("n,mltstp", [((16, 16, 16), 1), ((24, 20, 18), 1), ((15, 17, 9), 2)])
def test_esfield_matches_oracle(gpu, n, mltstp):
    c = case(n=n, ppc=(1, 1))
    cfg, eb, p, tp = build(c)
    rng = np.random.default_rng(sum(n))
    with Emses(cfg) as g:
        for mean in (0.0, 0.25):
            rho = rho_of(cfg, rng, mean)
            eb0 = rng.standard_normal(field_shape(cfg, "eb"))
            g.upload_field("rho", rho)
            g.upload_field("eb", eb0)
            res = g.esfield(mltstp)
            phi = g.download_field("phi").reshape(field_shape(cfg, "phi"))
            ebg = g.download_field("eb").reshape(field_shape(cfg, "eb"))
            phi_o, eb_o = E.esfield(rho, eb0, mltstp)
            e_phi = rel_l2(phi, phi_o)
            e_e = rel_l2(ebg[..., :3], eb_o[..., :3])
            print(f"{n} mean {mean}: phi {e_phi:.2e}, E {e_e:.2e}, poichk {res:.3e} "
                  f"(oracle {E.poichk(rho, phi_o):.3e})")
            assert e_phi < 1e-12 and e_e < 1e-12
            assert np.max(np.abs(phi - phi_o)) < 1e-12 * np.abs(phi_o).max()
            assert np.array_equal(ebg[..., 3:], eb0[..., 3:])
            # periodic guards copied exactly
            pz = phi[..., 0]
            assert np.array_equal(pz[0], pz[cfg.nz]) and np.array_equal(pz[cfg.nz + 2], pz[2])
            assert np.array_equal(pz[:, 0], pz[:, cfg.ny]) and np.array_equal(pz[:, :, cfg.nx + 1], pz[:, :, 1])
            want = abs(mean) / np.sqrt(cfg.nx * cfg.ny * cfg.nz)
            assert abs(res - want) < 1e-12 + 1e-9 * want


def test_es_loop_keeps_gauss_law(gpu):
    """The electrostatic loop on the FP32 form: a step, the field from its
    rho, the next step in that field; E's discrete divergence is the rho it
    came from (minus its mean) on every node."""
    c = case(n=(16, 16, 16), ppc=(8, 8), vth_scale=2.0, tile=(8, 8, 8))
    cfg, eb, p, tp = build(c)
    with Emses(cfg) as g:
        g.upload_particles(p, tp)
        g.upload_field("eb", eb)
        g.fx_load()
        for step in range(3):
            g.fx_step(2, step == 2)
            res = g.esfield(1)
            rho = g.download_field("rho").reshape(field_shape(cfg, "rho"))[..., 0]
            ebg = g.download_field("eb").reshape(field_shape(cfg, "eb"))
            nz, ny, nx = cfg.nz, cfg.ny, cfg.nx
            ex, ey, ez = ebg[..., 0], ebg[..., 1], ebg[..., 2]
            div = ((ex[1:nz + 1, 1:ny + 1, 1:nx + 1] - ex[1:nz + 1, 1:ny + 1, 0:nx])
                   + (ey[1:nz + 1, 1:ny + 1, 1:nx + 1] - ey[1:nz + 1, 0:ny, 1:nx + 1])
                   + (ez[1:nz + 1, 1:ny + 1, 1:nx + 1] - ez[0:nz, 1:ny + 1, 1:nx + 1]))
            r = rho[1:nz + 1, 1:ny + 1, 1:nx + 1]
            err = np.max(np.abs(div - (r - r.mean()))) / np.abs(r).max()
            print(f"step {step}: poichk {res:.3e}, div E - rho {err:.2e}")
            assert err < 1e-12


@pytest.mark.parametrize("mtd,n", [((1, 1, 1), (16, 16, 16)), ((0, 0, 1), (16, 12, 20)), ((2, 0, 0), (10, 12, 14)),
                                   ((1, 2, 0), (13, 16, 9)), ((2, 2, 2), (12, 12, 12)), ((0, 1, 2), (15, 10, 17))])
def test_esfield_faces_match_oracle(gpu, mtd, n):
    c = case(n=n, ppc=(1, 1))
    cfg, eb, p, tp = build(c)
    rng = np.random.default_rng(sum(n) + 10 * sum(mtd))
    bc = [tuple(rng.uniform(-0.5, 0.5, 2)) if mtd[d] == 2 else (0.0, 0.0) for d in range(3)]
    with Emses(cfg) as g:
        rho = rng.standard_normal(field_shape(cfg, "rho"))
        eb0 = rng.standard_normal(field_shape(cfg, "eb"))
        g.upload_field("rho", rho)
        g.upload_field("eb", eb0)
        res = g.esfield(2, mtd_vbnd=mtd, bc=bc)
        phi = g.download_field("phi").reshape(field_shape(cfg, "phi"))
        ebg = g.download_field("eb").reshape(field_shape(cfg, "eb"))
        phi_o, eb_o = E.esfield_general(rho, eb0, mtd, bc, mltstp=2)
        res_o = E.poichk_general(rho, phi_o, mtd)
        e_phi = rel_l2(phi, phi_o)
        e_e = rel_l2(ebg[..., :3], eb_o[..., :3])
        print(f"{mtd} {n}: phi {e_phi:.2e}, E {e_e:.2e}, poichk {res:.3e} (oracle {res_o:.3e})")
        assert e_phi < 1e-12 and e_e < 1e-12
        assert np.max(np.abs(phi - phi_o)) < 1e-12 * np.abs(phi_o).max()
        # zeros outside the solved nodes are exact
        assert np.array_equal(phi == 0.0, phi_o == 0.0)
        assert np.array_equal(ebg[..., 3:], eb0[..., 3:])
        assert abs(res - res_o) <= 1e-9 * max(res_o, 1e-300) + 1e-15
