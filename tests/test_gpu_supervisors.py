"""The injection supervisors on the device (emsesg_fx_emit,
emsesg_fx_inflow_z, emsesg_fx_inflow, emsesg_fx_emit_plane) against the host supervisors of ctca_b200/inject.py fed
the same counter-hash draws (inject.hash_uniforms): the injected records,
and everything downstream (the step's rho/J accumulators, the surface
counts, the particle records after the sort), are bit-identical."""
import numpy as np
import pytest

from ctca_b200 import inject, inputs, tables
from ctca_b200.emses import Emses

from helpers import build, case


@pytest.fixture
def trng():
    """The reference's random stream for the velocity tables of a test."""
    return tables.Ranu0(4357)

pytestmark = pytest.mark.gpu

BOX = dict(geotype=0, ncond=1, xlpc=8.0, xupc=16.0, ylpc=8.0, yupc=16.0, zlpc=14.0, zupc=18.0, sqdscaled=1.0)


def setup():
    c = case(n=(24, 24, 32), ppc=(3, 3), npbnd=(0, 0, 2), nfbnd=(0, 0, 1), vth_scale=3.0, tile=(8, 8, 8))
    for s in c.species:
        s.drift = (0.0, 0.0, -0.08)
    c.bodies = [BOX]
    cfg, eb, p, tp = build(c, capacity_factor=1.5)
    return c, cfg, eb


def loaded(c, cfg, eb):
    g = Emses(cfg)
    g.upload_field("eb", eb)
    g.fx_load_plasma(inputs.plasma(c, seed=5))
    return g


def test_device_supervisors_match_host(gpu, trng):
    c, cfg, eb = setup()
    renv = inputs.units()["renv"]
    vn = tables.signed_flux(512, 0.0, 0.01 * renv, 1, trng)[0]
    vt = tables.rann0(0.0, 0.01 * renv, 512, trng)
    s0 = c.species[0]
    vz = tables.signed_flux(512, -0.08 * renv, s0.vth * renv, -1, trng)[0]
    vx = tables.rann0(0.0, s0.vth * renv, 512, trng)
    vy = vx[::-1].copy()
    seed = 99
    with loaded(c, cfg, eb) as a, loaded(c, cfg, eb) as b:
        for step in range(3):
            ne, ni = 40 + step, 70 + 3 * step
            # host: the same draws as the device
            ue = inject.hash_uniforms(seed, 1, 1000 * step, ne, 6)
            ui = inject.hash_uniforms(seed, 2, 1000 * step, ni, 5)
            rec_e = inject.emit_rectangle(1, 16.0, (8.0, 16.0), (14.0, 18.0), ne, vn, vt, None, spec=1,
                                          uniforms=ue)
            rec_i = inject.inflow_z(False, ni, cfg.nx, cfg.ny, cfg.nz, vz, vx, vy, 2.0, None, spec=1, uniforms=ui)
            a.fx_inject(1, rec_e)
            a.fx_inject(1, rec_i)
            b.fx_emit(1, 1, 16.0, (8.0, 16.0), (14.0, 18.0), ne, vn, vt, seed, 1, 1000 * step)
            b.fx_inflow_z(1, False, ni, vz, vx, vy, 2.0, seed, 2, 1000 * step)
            a.fx_step(2, step == 1)
            b.fx_step(2, step == 1)
            ra, ja = a.fx_download_accum()
            rb, jb = b.fx_download_accum()
            assert np.array_equal(ra, rb), step
            assert np.array_equal(ja, jb), step
        assert np.array_equal(a.fx_surface(), b.fx_surface())
        assert np.abs(a.fx_surface()).sum() > 0
        a.fx_sort()
        b.fx_sort()
        a.fx_store()
        b.fx_store()
        pa, ta = a.download_particles()
        pb, tb = b.download_particles()
        assert np.array_equal(ta, tb)
        assert np.array_equal(pa.view(np.uint8), pb.view(np.uint8))


@pytest.mark.parametrize("axis", [0, 1])
def test_device_inflow_x_y_faces_match_host(gpu, axis, trng):
    """Inflow through both faces of x or y (open along that axis): device
    records against the host supervisor on the same draws, through a step
    and a sort."""
    npb = [0, 0, 0]
    npb[axis] = 2
    nfb = [0, 0, 0]
    nfb[axis] = 1
    c = case(n=(24, 16, 16), ppc=(3, 3), npbnd=tuple(npb), nfbnd=tuple(nfb), vth_scale=3.0, tile=(8, 8, 8))
    cfg, eb, p, tp = build(c, capacity_factor=1.5)
    renv = inputs.units()["renv"]
    s0 = c.species[0]
    va = tables.rann0(0.0, s0.vth * renv, 512, trng)
    vb = va[::-1].copy()
    ext = (cfg.nx, cfg.ny, cfg.nz)
    seed = 7
    with loaded(c, cfg, eb) as a, loaded(c, cfg, eb) as b:
        for step in range(2):
            for q, front in enumerate((True, False)):
                vn = tables.signed_flux(512, 0.0, s0.vth * renv, 1 if front else -1, trng)[0]
                n = 50 + 7 * step + q
                st = 10 + q
                u = inject.hash_uniforms(seed, st, 1000 * step, n, 5)
                rec = inject.inflow(axis, front, n, *ext, vn, va, vb, 2.0, None, spec=1, uniforms=u)
                a.fx_inject(1, rec)
                b.fx_inflow(1, axis, front, n, vn, va, vb, 2.0, seed, st, 1000 * step)
            a.fx_step(2, step == 1)
            b.fx_step(2, step == 1)
            ra, ja = a.fx_download_accum()
            rb, jb = b.fx_download_accum()
            assert np.array_equal(ra, rb), step
            assert np.array_equal(ja, jb), step
        a.fx_sort()
        b.fx_sort()
        a.fx_store()
        b.fx_store()
        pa, ta = a.download_particles()
        pb, tb = b.download_particles()
        assert np.array_equal(ta, tb)
        assert np.array_equal(pa.view(np.uint8), pb.view(np.uint8))


def test_device_plane_emission_matches_host(gpu, trng):
    """Plane emission (psuper2) from two planes inside a periodic box:
    device records against the host supervisor on the same draws, through
    steps and a sort."""
    c = case(n=(24, 24, 24), ppc=(3, 3), vth_scale=3.0, tile=(8, 8, 8))
    cfg, eb, p, tp = build(c, capacity_factor=1.5)
    renv = inputs.units()["renv"]
    vn = tables.signed_flux(512, 0.0, 0.01 * renv, 1, trng)[0]
    vt = tables.rann0(0.0, 0.01 * renv, 512, trng)
    seed = 31
    planes = [(1, 12.0, (4.0, 20.0), (6.0, 18.0), 1), (-3, 9.5, (2.0, 22.0), (3.0, 21.0), 2)]
    with loaded(c, cfg, eb) as a, loaded(c, cfg, eb) as b:
        for step in range(3):
            for q, (nemd, grd, b1, b2, pid) in enumerate(planes):
                n = 60 + 5 * step + q
                st = 20 + q
                u = inject.hash_uniforms(seed, st, 1000 * step, n, 6)
                rec = inject.emit_plane(nemd, grd, b1, b2, n, vn, vt, 2.0, None, spec=1, pid=pid, uniforms=u)
                a.fx_inject(1, rec)
                b.fx_emit_plane(1, nemd, grd, b1, b2, n, vn, vt, 2.0, pid, seed, st, 1000 * step)
            a.fx_step(2, step == 1)
            b.fx_step(2, step == 1)
            ra, ja = a.fx_download_accum()
            rb, jb = b.fx_download_accum()
            assert np.array_equal(ra, rb), step
            assert np.array_equal(ja, jb), step
        a.fx_sort()
        b.fx_sort()
        a.fx_store()
        b.fx_store()
        pa, ta = a.download_particles()
        pb, tb = b.download_particles()
        assert np.array_equal(ta, tb)
        assert np.array_equal(pa.view(np.uint8), pb.view(np.uint8))
