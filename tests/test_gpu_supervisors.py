"""The injection supervisors on the device (emsesg_fx_emit,
emsesg_fx_inflow_z, emsesg_fx_inflow, emsesg_fx_emit_plane) against the host supervisors of ctca_b200/inject.py fed
the same counter-hash draws (inject.hash_uniforms): the injected records,
and everything downstream (the step's rho/J accumulators, the surface
counts, the particle records after the sort), are bit-identical."""
import numpy as np
import pytest

from ctca_b200 import inject, inputs, tables
from ctca_b200.emses import Emses
from oracle import oracle as O

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


def test_device_cylinder_emission_matches_host(gpu, trng):
    """Emission from the end caps and the three kinds of side surface of
    cylinders along x, y and z (psuper3.F90:241-528): the device records
    against the host supervisor's on the same draws, both put into the FP32
    form (anti-particles dropped there) and given their first push.  The
    device's cos / sin may differ from the C library's in the last bit, so
    positions agree to 2 FP32 ulps of an in-cell offset and velocities to 2
    FP32 ulps; the counts and the order of the records are exact."""
    c = case(n=(24, 24, 24), ppc=(2, 2), vth_scale=3.0, tile=(8, 8, 8))
    cfg, eb, p, tp = build(c, capacity_factor=1.5)
    renv = inputs.units()["renv"]
    tabs = tables.emission_tables(512, 512, 0.0, 0.01 * renv, 0.01 * renv, 0.0, trng)
    seed = 77
    # (nemd, align, radius, axis, omni, grd, hl, hu, psi, anti)
    faces = [(3, 3, 4.5, (12.0, 11.5), 0, 18.0, 0.0, 0.0, 0.0, True),
             (-3, 3, 4.5, (12.0, 11.5), 0, 6.0, 0.0, 0.0, 0.0, False),
             (1, 3, 4.5, (12.0, 11.5), 0, 0.0, 6.0, 18.0, 0.3, True),
             (2, 3, 0.6, (12.0, 11.5), 0, 0.0, 6.0, 18.0, 0.3, True),
             (-1, 3, 4.5, (12.0, 11.5), 1, 0.0, 6.0, 18.0, 0.3, False),
             (1, 1, 3.0, (10.0, 13.0), 0, 17.0, 5.0, 17.0, 2.0, True),
             (2, 1, 3.0, (10.0, 13.0), 0, 0.0, 5.0, 17.0, 2.0, True),
             (3, 2, 2.5, (9.0, 14.0), 1, 0.0, 4.0, 20.0, 1.1, True)]
    with loaded(c, cfg, eb) as a, loaded(c, cfg, eb) as b:
        for q, (nemd, align, radius, axis, omni, grd, hl, hu, psi, anti) in enumerate(faces):
            n = 50 + 7 * q
            u = inject.hash_uniforms(seed, 40 + q, 0, n, 6).ravel()
            rec = inject.emit_cylinder(nemd, align, radius, axis, omni, grd, hl, hu, psi, n, tabs, None, spec=1,
                                       uniforms=u, anti=anti)
            a.fx_inject(1, rec)
            b.fx_emit_cylinder(1, nemd, align, radius, axis, omni, grd, hl, hu, psi, n, tabs, anti, seed, 40 + q)
        # the first (random, partial) push of the new particles, then the records
        a.fx_step(2, False)
        b.fx_step(2, False)
        assert np.array_equal(a.fx_counts(), b.fx_counts())
        a.fx_store()
        b.fx_store()
        pa, ta = a.download_particles()
        pb, tb = b.download_particles()
        assert np.array_equal(ta, tb)
        for f in ("pid", "preside", "nid", "spec"):
            assert np.array_equal(pa[f], pb[f]), f
        for f in ("x", "y", "z"):
            assert np.max(np.abs(pa[f] - pb[f])) <= 2 * 2.0 ** -24, f
        for f in ("vx", "vy", "vz"):
            assert np.max(np.abs(pa[f] - pb[f]) / np.maximum(np.abs(pa[f]), 1e-30)) <= 2 * 2.0 ** -23, f
        diff = sum(int(np.count_nonzero(pa[f] != pb[f])) for f in ("x", "y", "z", "vx", "vy", "vz"))
        print(f"cylinder emission: {ta.sum()} records, {diff} components differing in the last bits")


def test_device_inflow_current_matches_host(gpu, trng):
    """psuper1's injection current (psuper1.F90:120-323, current_deposition):
    the device deposits, into the J of the next step, the zigzag current of
    each inflow particle's path from outside the face; against the host
    supervisor's FP64 current (inject.inflow_current) times q, within the
    rounding of one 2^-40 fixed-point unit per contribution.  The step then
    adds its own deposit: J of the step equals that of the same particles
    injected without current plus the injection current, exactly."""
    c = case(n=(16, 16, 24), ppc=(3, 3), npbnd=(0, 0, 2), nfbnd=(0, 0, 1), vth_scale=3.0, tile=(8, 8, 8))
    cfg, eb, p, tp = build(c, capacity_factor=1.5)
    renv = inputs.units()["renv"]
    s0 = c.species[0]
    va = tables.rann0(0.0, s0.vth * renv, 512, trng)
    vb = tables.rann0(0.0, s0.vth * renv, 512, trng)
    ext = (cfg.nx, cfg.ny, cfg.nz)
    seed, ustep = 9, 2
    with loaded(c, cfg, eb) as a, loaded(c, cfg, eb) as b:
        wrk = np.zeros((ext[2] + 9, ext[1] + 9, ext[0] + 9, 3))
        ncontrib = 0
        for q, front in enumerate((True, False)):
            vn = tables.signed_flux(512, -0.02 * renv, s0.vth * renv, 1 if front else -1, trng)[0]
            n = 300 + 11 * q
            u = inject.hash_uniforms(seed, 30 + q, 0, n, 5)
            rec = inject.inflow(2, front, n, *ext, vn, va, vb, 2.0, None, spec=1, uniforms=u)
            inject.inflow_current(2, front, rec, ustep, ext, wrk)
            ncontrib += 24 * n
            a.fx_inject(1, rec)
            b.fx_inflow_current(1, 2, front, n, vn, va, vb, 2.0, ustep, seed, 30 + q, 0)
        _, jinj = b.fx_download_accum()
        want = wrk * cfg.q[0]
        got = jinj.astype(np.float64) * 2.0 ** -40
        err = np.max(np.abs(got - want))
        print(f"injection current: max |J| {np.max(np.abs(want)):.3e}, max error {err:.3e} "
              f"({ncontrib} contributions)")
        assert np.count_nonzero(want) > 0
        assert err <= ncontrib * 2.0 ** -41  # half a fixed-point unit per contribution, all at one node at worst
        a.fx_step(ustep, False)
        b.fx_step(ustep, False)
        ra, ja = a.fx_download_accum()
        rb, jb = b.fx_download_accum()
        assert np.array_equal(ra, rb)
        # the step folds the guard layers (add_boundary_current) of its J, an
        # integer-linear map: the difference is the folded injection current,
        # checked against the oracle's fold of the host's FP64 current
        o = O.Oracle(cfg, np.zeros(0, dtype=p.dtype), np.zeros(cfg.nspec, dtype=np.int64), eb)
        o.f["aj"][...] = want
        o.reduce_aj()
        folded = (jb - ja).astype(np.float64) * 2.0 ** -40
        ferr = np.max(np.abs(folded - o.f["aj"]))
        print(f"folded injection current: max error {ferr:.3e}")
        assert ferr <= ncontrib * 2.0 ** -41
        # the next step starts J from zero again
        a.fx_step(ustep, False)
        b.fx_step(ustep, False)
        assert np.array_equal(a.fx_download_accum()[1], b.fx_download_accum()[1])
