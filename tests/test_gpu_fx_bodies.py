"""The FP32 / fixed-point form with a conducting box body, an open z axis
with inflow through the back face, and photoelectron emission from the box's
+x face (a small copy of the body + inflow + emission workload), step by
step against the FP64 oracle started every step from the FP32 form's own
state with the same injected particles and random numbers
(ctca_b200/inject.py).

Every step: rho and J within 1e-5 relative L2 on the nodes 0..n, and the
step's absorbed counts per body (influx), escapes (nesc) and per-surface-cell
counts (absorbed minus emitted) equal to the oracle's.  A count may differ only by
particles this test lists as next to a decision FP32 rounding can flip: an
FP64 end point within four FP32 ulps of an integer plane (a cell, body or
outer face), or two body-face entry times within 1e-5 (the face crossed
last).  With none listed in a step, the counts must be equal.  At the end the
background charge from the surface counts (emsesg_fx_background) equals the
oracle's conversion of the same counts bit for bit."""
import ctypes

import numpy as np
import pytest

from ctca_b200 import inject, inputs, tables
from ctca_b200.emses import PARTICLE_DTYPE, Emses
from oracle import compare as C
from oracle import oracle as O

from helpers import build, case


@pytest.fixture
def trng():
    """The reference's random stream for the velocity tables of a test."""
    return tables.Ranu0(4357)

pytestmark = pytest.mark.gpu

BOX = dict(geotype=0, ncond=1, xlpc=8.0, xupc=16.0, ylpc=8.0, yupc=16.0, zlpc=14.0, zupc=18.0, sqdscaled=1.0)
BOUNDS = ((8, 8, 14), (16, 16, 18))


def inside(p):
    return ((p["x"] >= BOX["xlpc"]) & (p["x"] <= BOX["xupc"]) & (p["y"] >= BOX["ylpc"]) & (p["y"] <= BOX["yupc"])
            & (p["z"] >= BOX["zlpc"]) & (p["z"] <= BOX["zupc"]))


def with_injected(p, tp, batches):
    """The records p (species segments tp) with each species' injected
    records appended to its segment."""
    base = np.concatenate([[0], np.cumsum(tp)])
    parts, counts = [], []
    for s in range(len(tp)):
        seg = p[base[s]:base[s + 1]]
        rec = batches.get(s + 1)
        parts += [seg] + ([rec] if rec is not None else [])
        counts.append(seg.size + (rec.size if rec is not None else 0))
    return np.concatenate(parts).astype(PARTICLE_DTYPE), np.array(counts, dtype=np.int64)


def test_fx_box_inflow_emission_per_step(gpu, trng):
    c = case(n=(24, 24, 32), ppc=(4, 4), npbnd=(0, 0, 2), nfbnd=(0, 0, 1), vth_scale=3.0, tile=(8, 8, 8))
    for s in c.species:
        s.drift = (0.0, 0.0, -0.08)
    c.bodies = [BOX]
    cfg, eb, p, tp = build(c, capacity_factor=1.5)
    cfg.rng_mode = 1
    # no particle starts inside the body
    parts, counts = [], []
    base = np.concatenate([[0], np.cumsum(tp)])
    for s in range(cfg.nspec):
        seg = p[base[s]:base[s + 1]]
        seg = seg[~inside(seg)]
        parts.append(seg)
        counts.append(seg.size)
    p, tp = np.concatenate(parts), np.array(counts, dtype=np.int64)

    g = Emses(cfg)
    g.upload_particles(p, tp)
    g.upload_field("eb", eb)
    g.fx_load()
    g.fx_store()
    cur, tp_cur = g.download_particles()
    g.fx_load()
    rng = np.random.default_rng(77)
    uni = rng.random(200000)
    g.set_randoms(uni)
    drawn = 0

    renv = inputs.units()["renv"]
    vth = [s.vth * renv for s in c.species]
    vn = tables.signed_flux(1024, 0.0, 0.01 * renv, 1, trng)[0]
    vt = tables.rann0(0.0, 0.01 * renv, 1024, trng)
    inflow_tabs = [(tables.signed_flux(1024, -0.08 * renv, vth[s], -1, trng)[0], tables.rann0(0.0, vth[s], 1024, trng))
                   for s in range(2)]
    L = O.lib()
    surf_prev = g.fx_surface()
    gc_prev = g.get_counters().as_dict()
    totals = {"influx": 0, "nesc": 0, "emitted": 0, "listed": 0}
    for step in range(4):
        batches = {1: [], 2: []}
        batches[1].append(inject.emit_rectangle(1, 16.0, (8.0, 16.0), (14.0, 18.0), 40, vn, vt, rng, spec=1))
        for s in (1, 2):
            vz, vxy = inflow_tabs[s - 1]
            batches[s].append(inject.inflow_z(False, 60, cfg.nx, cfg.ny, cfg.nz, vz, vxy, vxy, 1.0, rng, spec=s))
        batches = {s: np.concatenate(b) for s, b in batches.items()}
        emitted = np.zeros_like(surf_prev)
        listed_anti = 0
        for s, rec in batches.items():
            g.fx_inject(s, rec)
            for r in rec[rec["preside"] == -2]:
                pt = (ctypes.c_double * 3)(r["x"], r["y"], r["z"])
                sc = L.orc_surface_point(ctypes.byref(cfg), 0, pt)
                assert sc >= 0
                emitted[s - 1, sc] += 1
                # an anti-particle next to a face-cell edge may count in the next cell
                fr = np.array([r["y"], r["z"]]) - np.floor([r["y"], r["z"]])
                listed_anti += int(np.any((fr < C.BAND) | (fr > 1 - C.BAND)))
        # the oracle starts from the FP32 form's state plus the same records
        start, tp_start = with_injected(cur, tp_cur, batches)
        o = O.Oracle(cfg, start, tp_start, eb)
        o.set_randoms(uni[drawn:])
        drawn += sum(int((r["preside"] == 1).sum()) for r in batches.values())
        o.grdcrt()
        o.f["aj"][...] = 0.0
        o.psolve1(2, 0)
        o.reduce_aj()
        o.charge(0)
        o.reduce_rho("rho")
        g.fx_step(2, True)  # the re-sort merges the injected particles
        assert C.field_errors(g.download_field("rho"), o.f["rho"], cfg)["l2_rel"] < 1e-5, step
        assert C.field_errors(g.download_field("aj"), o.f["aj"], cfg)["l2_rel"] < 1e-5, step
        # the step's counts
        # anti-particles sit on the body face by construction and never move:
        # they are listed above by their tangential coordinates
        near = C.near_faces(cfg, start, o.pbuf, bodies=[BOUNDS]) & (start["preside"] != -2)
        listed = np.flatnonzero(near)
        for m in listed:
            print(f"step {step}: listed particle {m} start ({start[m]['x']:.9f}, {start[m]['y']:.9f}, "
                  f"{start[m]['z']:.9f}) end ({o.pbuf[m]['x']:.9f}, {o.pbuf[m]['y']:.9f}, {o.pbuf[m]['z']:.9f})")
        nl = listed.size + listed_anti
        gc = g.get_counters().as_dict()
        og = o.gc.as_dict()
        d_influx = gc["influx"][:2, 0] - gc_prev["influx"][:2, 0]
        d_nesc = gc["nesc"][:2] - gc_prev["nesc"][:2]
        surf = g.fx_surface()
        d_surf = surf - surf_prev
        want_surf = o.surf[:, :surf.shape[1]] - emitted
        diff = (int(np.abs(d_influx - og["influx"][:2, 0]).sum()), int(np.abs(d_nesc - og["nesc"][:2]).sum()),
                int(np.abs(d_surf - want_surf).sum()))
        print(f"step {step}: influx {d_influx} (oracle {og['influx'][:2, 0]}), nesc {d_nesc} "
              f"(oracle {og['nesc'][:2]}), surface-count difference {diff[2]}, listed {nl}")
        assert diff[0] <= nl and diff[1] <= nl and diff[2] <= 2 * nl, (step, diff, nl)
        if nl == 0:
            assert diff == (0, 0, 0)
        totals["influx"] += int(og["influx"][:2, 0].sum())
        totals["nesc"] += int(og["nesc"][:2].sum())
        totals["emitted"] += int(emitted.sum())
        totals["listed"] += nl
        surf_prev, gc_prev = surf, gc
        g.fx_store()
        cur, tp_cur = g.download_particles()
    print("totals", totals)
    assert totals["influx"] > 20          # the box absorbed particles
    assert totals["nesc"] > 10            # particles left through the open z faces
    assert totals["emitted"] == 4 * 40
    # background charge from the counts, against the oracle's conversion
    rho = g.download_field("rho")
    g.fx_background(False)
    o2 = O.Oracle(cfg, cur[:0], [0, 0], eb)
    o2.f["rho"][...] = rho
    o2.background(surf=g.fx_surface())
    assert np.array_equal(g.download_field("rhobk"), o2.f["rhobk"])
    assert np.array_equal(g.download_field("rho"), o2.f["rho"])
    net = g.fx_surface().sum(1)
    assert abs(o2.f["rhobk"].sum() - sum(cfg.q[s] * net[s] for s in range(2))) < 1e-9 * abs(cfg.q[0]) * np.abs(net).sum()
    g.close()


# a box, a cylinder along x and a sphere, apart from each other, on a
# periodic 24^3 grid (the cylinder's axis and the sphere's centre off the
# cell nodes)
CURVED = [dict(geotype=0, ncond=1, xlpc=3.0, xupc=7.0, ylpc=3.0, yupc=7.0, zlpc=3.0, zupc=7.0, sqdscaled=1.0),
          dict(geotype=2, ncond=1, cyl_align=1, cyl_axis=(16.5, 8.25), cyl_edge=(2.0, 21.5), radius=3.3,
               sqdscaled=1.0),
          dict(geotype=3, ncond=0, sph_center=(15.3, 16.7, 17.1), radius=4.2)]


def inside_any(p, bodies):
    e = np.stack([p[f] for f in "xyz"], 1)
    m = np.zeros(p.size, dtype=bool)
    for b in bodies:
        if b["geotype"] in (0, 1):
            lo = np.array([b["xlpc"], b["ylpc"], b["zlpc"]])
            hi = np.array([b["xupc"], b["yupc"], b["zupc"]])
            m |= np.all((e >= lo) & (e <= hi), 1)
        elif b["geotype"] == 3:
            m |= ((e - np.asarray(b["sph_center"])) ** 2).sum(1) < b["radius"] ** 2
        else:
            a0 = b["cyl_align"] - 1
            a1, a2 = (a0 + 1) % 3, (a0 + 2) % 3
            d2 = (e[:, a1] - b["cyl_axis"][0]) ** 2 + (e[:, a2] - b["cyl_axis"][1]) ** 2
            m |= (e[:, a0] >= b["cyl_edge"][0]) & (e[:, a0] <= b["cyl_edge"][1]) & (d2 < b["radius"] ** 2)
    return m


@pytest.mark.parametrize("es", [False, True])
def test_fx_cylinder_sphere_per_step(gpu, es):
    """Cylinders and spheres in the FP32 form: every step from the FP32
    form's own state against the oracle, rho and J within 1e-5 relative L2
    and the absorbed counts of each body equal, except for particles listed
    as next to a decision FP32 rounding can flip (an end point within 1e-5
    cell of a curved surface, or next to an integer plane).  With `es` the
    step without the current against psolve2 + charge."""
    c = case(n=(24, 24, 24), ppc=(6, 6), vth_scale=3.0, tile=(8, 8, 8))
    c.bodies = CURVED
    cfg, eb, p, tp = build(c, capacity_factor=1.5)
    parts, counts = [], []
    base = np.concatenate([[0], np.cumsum(tp)])
    for s in range(cfg.nspec):
        seg = p[base[s]:base[s + 1]]
        seg = seg[~inside_any(seg, CURVED)]
        parts.append(seg)
        counts.append(seg.size)
    p, tp = np.concatenate(parts), np.array(counts, dtype=np.int64)
    g = Emses(cfg)
    g.upload_particles(p, tp)
    g.upload_field("eb", eb)
    g.fx_load()
    g.fx_store()
    cur, tp_cur = g.download_particles()
    gc_prev = g.get_counters().as_dict()
    totals = np.zeros(3, dtype=np.int64)
    listed_all = 0
    for step in range(4):
        o = O.Oracle(cfg, cur, tp_cur, eb)
        o.grdcrt()
        if es:
            o.psolve2(2)
        else:
            o.f["aj"][...] = 0.0
            o.psolve1(2, 0)
            o.reduce_aj()
        o.charge(0)
        o.reduce_rho("rho")
        if es:
            g.fx_step_es(2, step % 2 == 1)
        else:
            g.fx_step(2, step % 2 == 1)
        er = C.field_errors(g.download_field("rho"), o.f["rho"], cfg)["l2_rel"]
        ej = 0.0 if es else C.field_errors(g.download_field("aj"), o.f["aj"], cfg)["l2_rel"]
        live = cur["nid"] != -1  # records of particles that died since the last sort stay in place
        near = live & (C.near_faces(cfg, cur, o.pbuf, bodies=[((3, 3, 3), (7, 7, 7))])
                       | C.near_curved(o.pbuf, CURVED))
        nl = int(near.sum())
        gc = g.get_counters().as_dict()
        og = o.gc.as_dict()
        d_influx = gc["influx"][:2, :3] - gc_prev["influx"][:2, :3]
        diff = np.abs(d_influx - og["influx"][:2, :3])
        print(f"step {step}: rho {er:.2e}, J {ej:.2e}, influx {d_influx.sum(0)} (oracle {og['influx'][:2, :3].sum(0)}), "
              f"difference {int(diff.sum())}, listed {nl}")
        assert er < 1e-5 and ej < 1e-5, step
        assert int(diff.sum()) <= nl, step
        if nl == 0:
            assert int(diff.sum()) == 0
        # escapes: periodic, none
        assert int((gc["nesc"][:2] - gc_prev["nesc"][:2]).sum()) == 0
        totals += og["influx"][:2, :3].sum(0)
        listed_all += nl
        gc_prev = gc
        g.fx_store()
        cur, tp_cur = g.download_particles()
        # the absorbed particles are gone: what is left lies outside every body
        # (up to the listed band)
        left = (inside_any(cur, CURVED) & (cur["nid"] != -1) & ~C.near_curved(cur, CURVED)
                & ~C.near_faces(cfg, cur, cur))
        assert not left.any(), step
    print("absorbed per body", totals, "listed", listed_all)
    assert np.all(totals > 10)   # every body absorbed particles
    g.close()


def test_fx_load_plasma_leaves_out_curved_bodies(gpu):
    """The FP32 plasma loader places no particle inside a body (the push's
    absorption test), and places the same particles as the loader of the
    FP64 records outside them."""
    from ctca_b200 import inputs as I
    c = case(n=(24, 24, 24), ppc=(5, 5), tile=(8, 8, 8))
    c.bodies = CURVED
    cfg = I.make_config(c)
    eb = I.make_fields(c)
    pl = I.plasma(c, seed=9)
    with Emses(cfg) as a, Emses(cfg) as b:
        for g in (a, b):
            g.upload_field("eb", eb)
        a.load_plasma(pl)
        a.fx_load()
        a.fx_store()
        pa, ta = a.download_particles()
        b.fx_load_plasma(pl)
        b.fx_store()
        pb, tb = b.download_particles()
    pb = pb[pb["nid"] != -1]
    keep = ~inside_any(pa, CURVED)
    edge = C.near_curved(pa, CURVED) | C.near_faces(cfg, pa, pa)
    assert not (inside_any(pb, CURVED) & ~C.near_curved(pb, CURVED) & ~C.near_faces(cfg, pb, pb)).any()
    # the same particles outside the bodies (up to those on a surface)
    assert abs(int(pb.size) - int(keep.sum())) <= int(edge.sum())
    assert pb.size < pa.size


@pytest.mark.parametrize("es", [False, True])
def test_fx_particles_loaded_inside_a_box(gpu, es):
    """Records loaded with particles inside a box body (the reference's push
    absorbs every particle whose end point is inside, leaving its cell or
    not; a start point inside moves to the relay point, so the first zigzag
    segment carries no current): the first step of the FP32 form, with and
    without the current, absorbs the same particles as the oracle's
    psolve1 / psolve2 -- influx equal -- with rho and J within 1e-5."""
    c = case(n=(16, 16, 24), ppc=(8, 8), npbnd=(1, 0, 2), nfbnd=(1, 0, 1), vth_scale=3.0, tile=(8, 8, 8))
    c.bodies = [dict(geotype=0, ncond=1, xlpc=3.0, xupc=7.0, ylpc=3.0, yupc=7.0, zlpc=4.0, zupc=9.0, sqdscaled=1.0)]
    cfg, eb, p, tp = build(c, 1.2)
    g = Emses(cfg)
    g.upload_particles(p, tp)
    g.upload_field("eb", eb)
    g.fx_load()
    g.fx_store()
    p32, tp32 = g.download_particles()
    g.fx_load()
    o = O.Oracle(cfg, p32, tp32, eb)
    o.grdcrt()
    if es:
        o.psolve2(2)
    else:
        o.f["aj"][...] = 0.0
        o.psolve1(2, 0)
        o.reduce_aj()
    o.charge(0)
    o.reduce_rho("rho")
    if es:
        g.fx_step_es(2, False)
    else:
        g.fx_step(2, False)
    gi = g.get_counters().as_dict()["influx"][:2, 0]
    oi = o.gc.as_dict()["influx"][:2, 0]
    print("influx", gi, "oracle", oi)
    assert oi.sum() > 100 and np.array_equal(gi, oi)
    assert C.field_errors(g.download_field("rho"), o.f["rho"], cfg)["l2_rel"] < 1e-5
    if not es:
        assert C.field_errors(g.download_field("aj"), o.f["aj"], cfg)["l2_rel"] < 1e-5
    g.close()
