"""Host-side injection supervisors (ctca_b200/inject.py) and the oracle's
surface-cell rule of the box bodies."""
import ctypes
import math

import numpy as np
import pytest

from ctca_b200 import inject, inputs, tables
from oracle import oracle as O

from helpers import case


@pytest.fixture
def trng():
    """The reference's random stream for the velocity tables of a test."""
    return tables.Ranu0(4357)


def test_flux_tables(trng):
    """The reference's tables (ctca_b200/tables.py, pinned bit for bit by
    test_golden_tables.py) have the moments of their distributions."""
    vth, npr = 0.3, 4000
    r = tables.signed_flux(npr, 0.0, vth, 1, trng)[0]
    assert np.all(r > 0)
    # flux of a Maxwellian: Rayleigh (the mid-point steps of vflux end short
    # of the far tail: 0.2 % low at 4000 entries)
    assert abs(r.mean() - vth * math.sqrt(math.pi / 2)) < 5e-3 * vth
    t = tables.rann0(0.1, vth, npr, trng)
    assert abs(t.mean() - 0.1) < 4 * vth / math.sqrt(npr) and abs(t.std() - vth) < 0.05 * vth
    # drifting flux toward -z: all negative, faster than the drift on average
    b = tables.signed_flux(npr, -0.5, vth, -1, trng)[0]
    assert np.all(b < 0) and b.mean() < -0.5


def test_emission_count_matches_the_reference_formula():
    # (int((istep+lstep)*fluxf) - int((istep+lstep-injct)*fluxf)) * ustep
    assert inject.emission_count(10, 0, 3.7, 1, 2) == (int(10 * 3.7) - int(9 * 3.7)) * 2
    assert sum(inject.emission_count(s, 0, 0.25, 1, 1) for s in range(1, 9)) == 2


def test_emit_rectangle_pairs(trng):
    rng = np.random.default_rng(3)
    vn = tables.signed_flux(256, 0.0, 0.01, 1, trng)[0]
    vt = tables.rann0(0.0, 0.01, 256, trng)
    for nemd, ax in ((1, "x"), (-2, "y"), (3, "z")):
        rec = inject.emit_rectangle(nemd, 16.0, (8.0, 16.0), (14.0, 18.0), 50, vn, vt, rng, spec=1)
        anti, twin = rec[0::2], rec[1::2]
        assert np.all(anti["preside"] == -2) and np.all(twin["preside"] == 1)
        assert np.all(anti[ax] == 16.0)
        assert np.allclose(twin[ax] - anti[ax], np.sign(nemd) * 1e-5)
        assert np.all(np.sign(twin["v" + ax]) == np.sign(nemd))
        for c in "xyz":
            if c != ax:
                assert np.array_equal(anti[c], twin[c])


def test_inflow_positions(trng):
    rng = np.random.default_rng(4)
    vz = tables.signed_flux(512, -0.08, 0.05, -1, trng)[0]
    vx = tables.rann0(0.0, 0.05, 512, trng)
    rec = inject.inflow_z(False, 1000, 24, 24, 32, vz, vx, vx, 1.0, rng, spec=1)
    assert np.all(rec["z"] <= 32) and np.all(rec["z"] >= 32 + vz.min())
    assert np.all(rec["vz"] < 0) and np.all(rec["preside"] == 0)
    assert np.all((rec["x"] >= 0) & (rec["x"] < 24))


@pytest.mark.parametrize("axis", [0, 1, 2])
@pytest.mark.parametrize("front", [True, False])
def test_inflow_faces(axis, front, trng):
    """Inflow through every face (psuper2.F90:114-292): the normal coordinate
    within vn * injctisw of the face, the tangential ones uniform on it, the
    normal speed from the normal table and the tangential ones from one draw
    of the tangential tables; the z faces are inflow_z."""
    ext = (24, 20, 32)
    names = "xyz"
    sgn = 1.0 if front else -1.0
    vn = tables.signed_flux(512, 0.0, 0.05, int(sgn), trng)[0]
    va = tables.rann0(0.0, 0.05, 512, trng)
    vb = va[::-1].copy()
    u = inject.hash_uniforms(3, 4, 0, 2000, 5)
    rec = inject.inflow(axis, front, 2000, *ext, vn, va, vb, 2.0, None, spec=2, uniforms=u)
    assert rec.size == 2000 and np.all(rec["spec"] == 2) and np.all(rec["preside"] == 0)
    n = names[axis]
    depth = rec[n] if front else rec[n] - ext[axis]
    assert np.all(sgn * depth >= 0) and np.all(np.abs(depth) <= 2.0 * np.abs(vn).max())
    assert np.allclose(depth, rec["v" + n] * 2.0 * u[:, 2 + axis])
    tang = [d for d in range(3) if d != axis]
    for d in tang:
        assert np.all((rec[names[d]] >= 0) & (rec[names[d]] < ext[d]))
        assert np.array_equal(rec[names[d]], 0.0 + ext[d] * u[:, 2 + d])
    a2 = (512 * u[:, 1]).astype(np.int64)
    assert np.array_equal(rec["v" + names[tang[0]]], va[a2])
    assert np.array_equal(rec["v" + names[tang[1]]], vb[a2])
    if axis == 2:
        z = inject.inflow_z(front, 2000, *ext, vn, va, vb, 2.0, None, spec=2, uniforms=u)
        assert np.array_equal(z.view(np.uint8), rec.view(np.uint8))


@pytest.mark.parametrize("nemd", [1, -1, 2, -2, 3, -3])
def test_emit_plane_geometry(nemd, trng):
    """Plane emission (emit_from_rectangular_surf, psuper2.F90:554-576):
    one record per particle with preside 0 and pid of the body; the normal
    coordinate grd + vnorm * injctisw * u3 on the side of nemd, the tangential
    ones uniform on the plane plus vtang * injctisw * u3."""
    vn_t = tables.signed_flux(256, 0.0, 0.01, 1, trng)[0]
    vt_t = tables.rann0(0.0, 0.01, 256, trng)
    u = inject.hash_uniforms(5, 6, 0, 500, 6)
    b1, b2 = (8.0, 16.0), (14.0, 18.0)
    rec = inject.emit_plane(nemd, 16.0, b1, b2, 500, vn_t, vt_t, 2.0, None, spec=1, pid=3, uniforms=u)
    assert rec.size == 500 and np.all(rec["preside"] == 0) and np.all(rec["pid"] == 3)
    ax = inject._ORDER[abs(nemd)]
    names = "xyz"
    n0, t1, t2 = (names[a] for a in ax)
    sgn = 1.0 if nemd > 0 else -1.0
    a0 = (256 * u[:, 0]).astype(np.int64)
    assert np.array_equal(rec["v" + n0], sgn * vn_t[a0])
    assert np.all(sgn * (rec[n0] - 16.0) >= 0)
    assert np.allclose(rec[n0], 16.0 + rec["v" + n0] * 2.0 * u[:, 3])
    for t, (lo, hi), c in ((t1, b1, 4), (t2, b2, 5)):
        on_plane = rec[t] - rec["v" + t] * 2.0 * u[:, 3]
        assert np.allclose(on_plane, lo + (hi - lo) * u[:, c])


def _box_cfg():
    c = case(n=(24, 24, 32))
    c.bodies = [dict(geotype=0, ncond=1, xlpc=8.0, xupc=16.0, ylpc=8.0, yupc=16.0, zlpc=14.0, zupc=18.0,
                     sqdscaled=1.0)]
    return inputs.make_config(c)


def test_surface_layout_and_rule():
    cfg = _box_cfg()
    L = O.lib()
    off = (ctypes.c_int64 * (6 * 15))()
    n = L.orc_surface_layout(ctypes.byref(cfg), off)
    # x faces 8x4, y faces 8x4, z faces 8x8
    assert n == 2 * 32 + 2 * 32 + 2 * 64
    assert list(off[:6]) == [0, 32, 64, 96, 128, 192]

    def cell(b, a):
        bb = (ctypes.c_double * 3)(*b)
        aa = (ctypes.c_double * 3)(*a)
        return L.orc_surface_cell(ctypes.byref(cfg), 0, bb, aa)

    # through the +x face (x = 16) into cell y=10, z=15
    assert cell((16.3, 10.5, 15.5), (15.8, 10.5, 15.5)) == 32 + (10 - 8) + 8 * (15 - 14)
    # through the -z face (z = 14) at x=9, y=12
    assert cell((9.5, 12.2, 13.9), (9.5, 12.2, 14.1)) == 128 + (9 - 8) + 8 * (12 - 8)
    # corner: crosses x = 8 at t = 0.75, z = 14 at t = 0.5: the x face is crossed last
    assert cell((7.7, 9.5, 13.8), (8.1, 9.5, 14.2)) == 0 + (9 - 8) + 8 * (14 - 14)
    p = (ctypes.c_double * 3)(16.0, 11.25, 17.5)
    assert L.orc_surface_point(ctypes.byref(cfg), 0, p) == 32 + 3 + 8 * 3
