"""CUDA-graph replay of the FP32 form and the ensemble batch.

A step replayed from a graph runs the same kernels on the same buffers as
emsesg_fx_step, so rho/J accumulators and particle records must come out
bit-identical to the step-by-step run.  A tile sort inside a graph that
meets a particle outside its tile's sort box keeps the current order
instead of the global sort: the particles (compared as a set) stay
bit-identical and rho/J agree to FP32 summation order."""
import numpy as np
import pytest

from ctca_b200 import ensemble, inputs
from ctca_b200.emses import Batch, Emses

from helpers import build, case, rel_l2

pytestmark = pytest.mark.gpu


def loaded(c, p=None, tp=None):
    cfg, eb, p0, tp0 = build(c, 1.2)
    if p is None:
        p, tp = p0, tp0
    g = Emses(cfg)
    g.upload_particles(p, tp)
    g.upload_field("eb", eb)
    g.fx_load()
    return g


def state(g):
    rho, j = g.fx_download_accum()
    g.fx_store()
    p, tp = g.download_particles()
    return rho, j, p, tp


def as_set(p):
    keys = np.stack([p[f] for f in ("x", "y", "z", "vx", "vy", "vz")])
    return p[np.lexsort(keys)]


@pytest.mark.parametrize("sort_every,nsteps", [(1, 7), (2, 12), (4, 8)])
def test_fx_run_graph_is_bit_identical_to_steps(gpu, sort_every, nsteps):
    c = case(n=(16, 16, 16), ppc=(8, 8), vth_scale=2.0, tile=(8, 8, 8))
    with loaded(c) as a, loaded(c) as b:
        a.fx_run(2, nsteps, sort_every, use_graph=False)
        b.fx_run(2, nsteps, sort_every, use_graph=True)
        b.fx_run(2, nsteps, sort_every, use_graph=True)  # replays the cached graph
        a.fx_run(2, nsteps, sort_every, use_graph=False)
        a.synchronize()
        b.synchronize()
        ra, ja, pa, ta = state(a)
        rb, jb, pb, tb = state(b)
        assert np.array_equal(ta, tb)
        assert np.array_equal(ra, rb)
        assert np.array_equal(ja, jb)
        assert np.array_equal(pa.view(np.uint8), pb.view(np.uint8))


def test_batch_is_bit_identical_to_each_run(gpu):
    cases = [case(n=(16, 16, 16), ppc=(8, 6), seed=3, tile=(8, 8, 8)),
             case(n=(24, 24, 24), ppc=(5, 7), seed=4, tile=(4, 4, 4), b0=(0.1, 0.0, 0.1)),
             case(n=(8, 16, 24), ppc=(9, 4), seed=5, tile=(8, 8, 8), vth_scale=2.0)]
    sorts = [1, 2, 4]
    block = ensemble.block_steps(sorts)
    assert block == 8
    solo = [loaded(c) for c in cases]
    many = [loaded(c) for c in cases]
    try:
        for g, s in zip(solo, sorts):
            g.fx_run(2, 2 * block, s, use_graph=False)
        with Batch(many, 2, block, sorts) as b:
            b.launch(2)
        for g, h in zip(solo, many):
            g.synchronize()
            h.synchronize()
            r1, j1, p1, t1 = state(g)
            r2, j2, p2, t2 = state(h)
            assert np.array_equal(t1, t2)
            assert np.array_equal(r1, r2)
            assert np.array_equal(j1, j2)
            assert np.array_equal(p1.view(np.uint8), p2.view(np.uint8))
    finally:
        for g in solo + many:
            g.close()


def test_batch_rejects_bad_block(gpu):
    c = case(n=(16, 16, 16), ppc=(4, 4), tile=(8, 8, 8))
    with loaded(c) as g:
        with pytest.raises(Exception, match="multiple of 2"):
            Batch([g], 2, 6, [4])


def test_graph_sort_with_a_stray_keeps_order(gpu):
    # one fast electron crosses 0.9 cells per step: after 4 steps it has
    # left its tile's sort box (tile + 1 cell), so the eager run falls back
    # to the global sort while the graph keeps the order
    c = case(n=(16, 16, 16), ppc=(4, 4), tile=(4, 4, 4), e=False, b0=(0.0, 0.0, 0.0))
    cfg, eb, p, tp = build(c, 1.2)
    p = p.copy()
    p["vx"][0] = 0.45
    p["vy"][0] = 0.0
    p["vz"][0] = 0.0
    with loaded(c, p, tp) as a, loaded(c, p, tp) as b:
        a.fx_run(2, 8, 4, use_graph=False)
        b.fx_run(2, 8, 4, use_graph=True)
        a.synchronize()
        b.synchronize()
        ra, ja, pa, ta = state(a)
        rb, jb, pb, tb = state(b)
        assert np.array_equal(ta, tb)
        sa, sb = as_set(pa), as_set(pb)
        assert np.array_equal(sa.view(np.uint8), sb.view(np.uint8))
        assert rel_l2(rb, ra) < 1e-6
        assert rel_l2(jb, ja) < 1e-6
        # the graph run keeps going from its unsorted state
        b.fx_run(2, 8, 4, use_graph=True)
        a.fx_run(2, 8, 4, use_graph=False)
        a.synchronize()
        b.synchronize()
        ra, ja, pa, _ = state(a)
        rb, jb, pb, _ = state(b)
        assert np.array_equal(as_set(pa).view(np.uint8), as_set(pb).view(np.uint8))
        assert rel_l2(rb, ra) < 1e-6
        assert rel_l2(jb, ja) < 1e-6


def test_small_ensemble_runs_and_tunes(gpu):
    cases = ensemble.ensemble_cases(6, seed=77, sides=(16, 24))
    for c in cases:
        for s in c.species:
            s.ppc = min(s.ppc, 12)
    tuner = ensemble.Autotuner(steps=4, trial_particles=1 << 20)
    out = ensemble.run_ensemble(cases, 16, tuner, modes=("batch", "each", "each_graph"), warm=2)
    assert out["particle_steps"] == 16 * sum(ensemble.particles(c) for c in cases)
    for m in ("batch", "each", "each_graph"):
        assert out["particle_steps_per_s"][m] > 0
    assert out["batch_kernels"] > 0
    assert out["e2e_seconds"] > out["seconds"]["batch"]
    assert set(out["choices"]) <= {"side16", "side24"}
    for ch in out["choices"].values():
        assert ch["tile"] in ensemble.TILES and ch["sort_every"] in ensemble.SORTS
        assert ch["chunk_rows"] in ensemble.CHUNKS


@pytest.mark.parametrize("rows", [1, 16, 48])
def test_rows_per_cta_change_no_particle(gpu, rows):
    """Fewer rows of a tile region per push CTA (the autotuner's block
    knob): several CTAs share a tile, so a thread's run sums split at the
    chunk edges; the particles stay bit-identical and rho / J agree to FP32
    summation order."""
    c = case(n=(16, 16, 16), ppc=(24, 24), vth_scale=2.0, tile=(8, 8, 8))
    with loaded(c) as a, loaded(c) as b:
        b.fx_chunk_rows(rows)
        a.fx_run(2, 8, 4, use_graph=False)
        b.fx_run(2, 8, 4, use_graph=False)
        ra, ja, pa, ta = state(a)
        rb, jb, pb, tb = state(b)
        assert np.array_equal(ta, tb)
        assert np.array_equal(pa.view(np.uint8), pb.view(np.uint8))
        assert rel_l2(rb, ra) < 1e-6 and rel_l2(jb, ja) < 1e-6
