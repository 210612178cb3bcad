"""The z-slab decomposition of the FP32 form (ctca_b200/slabs.py, slab mode
of libemsesg) against one context holding the whole grid.

The first step is exact: a slab's push deposits the same int64
contributions as the whole grid's (the slabs' tiles are the whole grid's
tiles, so the same particles share the same runs), the particles that leave
a slab carry their current in its guard planes and have their charge
deposited by the slab they enter, and the exchange of the z border planes
followed by the guard folds adds them up as the whole grid's periodic fold
does.  rho and J on every node, the counts and the particles are then equal
bit for bit.  Later steps push the particles that changed slab on the tail
path (global field gather, IEEE division) instead of the tile path, so their
FP32 values may differ in the last bits: over 8 steps with two re-sorts rho
and J stay within 1e-5 relative L2 and the particle counts are exact."""
import numpy as np
import pytest

from ctca_b200 import slabs
from ctca_b200.emses import Emses, field_extents, field_shape

from helpers import build, case, rel_l2

pytestmark = pytest.mark.gpu

OUTBOX = 40000


def whole_nodes(cfg, a, name):
    nc, lo, ex, ey, ez = field_extents(cfg, name)
    a = a.reshape(field_shape(cfg, name)[:3] + (nc,))
    return a[-lo:-lo + cfg.nz + 1, -lo:-lo + cfg.ny + 1, -lo:-lo + cfg.nx + 1]


def setup(nz=32, ppc=(4, 4)):
    c = case(n=(16, 16, nz), ppc=ppc, vth_scale=4.0, tile=(8, 8, 8))
    return build(c, capacity_factor=1.5)


def sorted_records(recs):
    keys = np.lexsort((recs["vz"], recs["vy"], recs["vx"], recs["z"], recs["y"], recs["x"], recs["spec"]))
    return recs[keys]


@pytest.mark.parametrize("nslab", [1, 2, 4])
def test_slab_first_step_exact(gpu, nslab):
    cfg, eb, p, tp = setup()
    with Emses(cfg) as w, slabs.SlabGroup(cfg, eb, p, tp, nslab, OUTBOX) as grp:
        w.upload_particles(p, tp)
        w.upload_field("eb", eb)
        w.fx_load()
        w.fx_step(2, False)
        grp.step(2, False)
        print(f"{nslab} slabs: {grp.migrated} particles changed slab")
        if nslab > 1:
            assert grp.migrated > 0
        for name in ("rho", "aj"):
            got = grp.fields(name)
            want = whole_nodes(cfg, w.download_field(name), name)
            assert np.array_equal(got, want), name
        assert np.array_equal(grp.counts(), w.fx_counts())
        # the particles: the slabs' records, shifted back, are the whole
        # grid's (as multisets)
        w.fx_store()
        pw, tw = w.download_particles()
        parts = []
        for r, g in enumerate(grp.ctx):
            g.fx_sort()  # merges the arrivals of the tail zone
            g.fx_store()
            pr, tr = g.download_particles()
            pr = pr.copy()
            pr["z"] += r * (cfg.nz // nslab)
            parts.append(pr)
        pg = np.concatenate(parts)
        assert pg.size == pw.size
        a, b = sorted_records(pg), sorted_records(pw)
        for f in ("x", "y", "z", "vx", "vy", "vz", "spec"):
            assert np.array_equal(a[f], b[f]), f


@pytest.mark.parametrize("nslab", [2, 4])
def test_slab_steps_close(gpu, nslab):
    cfg, eb, p, tp = setup()
    with Emses(cfg) as w, slabs.SlabGroup(cfg, eb, p, tp, nslab, OUTBOX) as grp:
        w.upload_particles(p, tp)
        w.upload_field("eb", eb)
        w.fx_load()
        for step in range(8):
            srt = step % 4 == 3
            w.fx_step(2, srt)
            grp.step(2, srt)
            er = rel_l2(grp.fields("rho"), whole_nodes(cfg, w.download_field("rho"), "rho"))
            ej = rel_l2(grp.fields("aj"), whole_nodes(cfg, w.download_field("aj"), "aj"))
            print(f"{nslab} slabs, step {step}: rho {er:.2e}, J {ej:.2e}, changed slab so far {grp.migrated}")
            assert er < 1e-5 and ej < 1e-5, step
            assert np.array_equal(grp.counts(), w.fx_counts()), step
