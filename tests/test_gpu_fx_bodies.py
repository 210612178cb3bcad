"""The FP32 / fixed-point form with a conducting box body, an open z axis
with inflow through the back face, and photoelectron emission from the box's
+x face: a small copy of the body + inflow + emission workload, against the
FP64 oracle run on the same FP32-rounded start state and the same injected
particles (ctca_b200/inject.py) and random numbers.

Checked every step: rho and J within 1e-5 relative L2.  At the end: the
absorbed counts per body (influx), the escape counts (nesc) and the
per-surface-cell counts (absorbed minus emitted) agree, up to one particle
that FP32 rounding may put on the other side of a face."""
import ctypes

import numpy as np
import pytest

from ctca_b200 import inject, inputs
from ctca_b200.emses import PARTICLE_DTYPE, Counter, Emses
from oracle import oracle as O

from helpers import build, case, rel_l2

pytestmark = pytest.mark.gpu

BOX = dict(geotype=0, ncond=1, xlpc=8.0, xupc=16.0, ylpc=8.0, yupc=16.0, zlpc=14.0, zupc=18.0, sqdscaled=1.0)


def inside(p):
    return ((p["x"] >= BOX["xlpc"]) & (p["x"] <= BOX["xupc"]) & (p["y"] >= BOX["ylpc"]) & (p["y"] <= BOX["yupc"])
            & (p["z"] >= BOX["zlpc"]) & (p["z"] <= BOX["zupc"]))


def oracle_inject(o, spec, rec):
    base = np.concatenate([[0], np.cumsum(o.totalp)])
    end = int(base[spec])
    o.pbuf = np.concatenate([o.pbuf[:end], rec, o.pbuf[end:]]).astype(PARTICLE_DTYPE)
    o.totalp[spec - 1] += rec.size


def test_fx_box_inflow_emission_vs_oracle(gpu):
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
    p32, tp32 = g.download_particles()
    g.fx_load()
    o = O.Oracle(cfg, p32, tp32, eb)
    rng = np.random.default_rng(77)
    uni = rng.random(200000)
    g.set_randoms(uni)
    o.set_randoms(uni)

    renv = inputs.units()["renv"]
    vth = [s.vth * renv for s in c.species]
    vn = inject.flux_table(0.01 * renv, 0.0, 1024)
    vt = inject.maxwell_table(0.01 * renv, 0.0, 1024)
    inflow_tabs = [(inject.flux_table(vth[s], -0.08 * renv, 1024, sign=-1.0), inject.maxwell_table(vth[s], 0.0, 1024))
                   for s in range(2)]
    emitted = np.zeros_like(o.surf)
    L = O.lib()
    for step in range(3):
        batches = {1: [], 2: []}
        batches[1].append(inject.emit_rectangle(1, 16.0, (8.0, 16.0), (14.0, 18.0), 40, vn, vt, rng, spec=1))
        for s in (1, 2):
            vz, vxy = inflow_tabs[s - 1]
            batches[s].append(inject.inflow_z(False, 60, cfg.nx, cfg.ny, cfg.nz, vz, vxy, vxy, 1.0, rng, spec=s))
        for s in (1, 2):
            rec = np.concatenate(batches[s])
            g.fx_inject(s, rec)
            oracle_inject(o, s, rec)
            for r in rec[rec["preside"] == -2]:
                pt = (ctypes.c_double * 3)(r["x"], r["y"], r["z"])
                sc = L.orc_surface_point(ctypes.byref(cfg), 0, pt)
                assert sc >= 0
                emitted[s - 1, sc] += 1
        g.fx_step(2, step == 1)
        o.grdcrt()
        o.f["aj"][...] = 0.0
        o.psolve1(2, 0)
        o.reduce_aj()
        o.charge(0)
        o.reduce_rho("rho")
        assert rel_l2(g.download_field("rho"), o.f["rho"]) < 1e-5, step
        assert rel_l2(g.download_field("aj"), o.f["aj"]) < 1e-5, step

    gc = g.get_counters().as_dict()
    og = o.gc.as_dict()
    assert og["influx"][:2, 0].sum() > 20          # the box absorbed particles
    assert np.all(np.abs(gc["influx"] - og["influx"]) <= 1)
    assert np.all(np.abs(gc["nesc"] - og["nesc"]) <= 1)
    assert og["nesc"][:2].sum() > 10               # particles left through the open z faces
    surf = g.fx_surface()
    want = o.surf[:, :surf.shape[1]] - emitted[:, :surf.shape[1]]
    assert surf.shape == (2, o.nsurf)
    assert np.abs(surf - want).sum() <= 2
    assert abs(surf.sum() - want.sum()) <= 1
    assert (emitted.sum() == 3 * 40)
    g.close()
