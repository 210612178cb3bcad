"""Parity of the plain FP64 GPU drop-in with the oracle, through the C ABI.

Bit-exact: particle records after grdcrt/psolve2/psolve1 (compiled without
FMA contraction), counters, sort permutation, compaction, guard folds and
rhoupd on identical inputs.  Within 1e-12 relative: rho / J / energy, whose
FP64 sums are formed by atomics in another order than the reference's
particle loop."""
import numpy as np
import pytest

from ctca_b200.emses import Counter, Emses
from oracle import oracle as O

from helpers import build, case, rel_l2, same_particles

pytestmark = pytest.mark.gpu

TOL = 1e-12  # FP64 summation-order tolerance for rho, J, energy


def pair(c, capacity_factor=1.0):
    cfg, eb, p, tp = build(c, capacity_factor)
    g = Emses(cfg)
    g.upload_particles(p, tp)
    g.upload_field("eb", eb)
    o = O.Oracle(cfg, p, tp, eb)
    return cfg, g, o


def counters_equal(a: Counter, b: Counter):
    da, db = a.as_dict(), b.as_dict()
    for k in ("influx", "infhist", "nesc"):
        assert np.array_equal(da[k], db[k]), k
    assert np.array_equal(da["chgacm"], db["chgacm"])


def test_grdcrt_bit_exact(gpu):
    cfg, g, o = pair(case(n=(8, 6, 10)))
    g.grdcrt(1)
    o.grdcrt()
    w = g.download_field("wrk")
    # nodes 0..n of EX..BZ
    sl = (slice(4, 4 + cfg.nz + 1), slice(4, 4 + cfg.ny + 1), slice(4, 4 + cfg.nx + 1), slice(0, 6))
    assert np.array_equal(w[sl], o.f["wrk"][sl])


@pytest.mark.parametrize("npbnd", [(0, 0, 0), (1, 1, 1), (2, 2, 2), (0, 1, 2)])
def test_psolve2_bit_exact(gpu, npbnd):
    c = case(npbnd=npbnd, vth_scale=4.0)
    c.bodies = [dict(geotype=0, ncond=1, xlpc=3.0, xupc=5.0, ylpc=2.5, yupc=5.5, zlpc=3.0, zupc=4.0, sqdscaled=0.5),
                dict(geotype=2, ncond=1, cyl_align=3, cyl_axis=(1.5, 6.0), cyl_edge=(1.0, 7.0), radius=0.8,
                     sqdscaled=0.25),
                dict(geotype=3, ncond=0, sph_center=(6.0, 2.0, 6.0), radius=1.1)]
    cfg, g, o = pair(c)
    g.grdcrt(1)
    o.grdcrt()
    gc = Counter()
    for _ in range(3):
        g.psolve2(1, 2, gc)
        o.psolve2(2)
        counters_equal(gc, o.gc)
    pg, tpg = g.download_particles()
    assert np.array_equal(tpg, o.totalp)
    assert same_particles(pg, o.pbuf)


@pytest.mark.parametrize("npbnd,nfbnd", [((0, 0, 0), (0, 0, 0)), ((1, 1, 1), (1, 1, 1)), ((0, 0, 2), (0, 0, 1))])
def test_psolve1_particles_exact_current_close(gpu, npbnd, nfbnd):
    c = case(npbnd=npbnd, nfbnd=nfbnd, vth_scale=4.0)
    c.bodies = [dict(geotype=1, ncond=1, xlpc=3.0, xupc=5.0, ylpc=3.0, yupc=5.0, zlpc=3.0, zupc=5.0, sqdscaled=1.0)]
    cfg, g, o = pair(c)
    g.grdcrt(1)
    o.grdcrt()
    gc = Counter()
    g.zero_field("aj")
    g.zero_field("ajdg")
    g.psolve1(1, 2, 1, gc)
    o.psolve1(2, 1)
    counters_equal(gc, o.gc)
    pg, _ = g.download_particles()
    assert same_particles(pg, o.pbuf)
    assert rel_l2(g.download_field("aj"), o.f["aj"]) < TOL
    assert rel_l2(g.download_field("ajdg"), o.f["ajdg"]) < TOL
    g.reduce_aj()
    o.reduce_aj()
    g.reduce_ajdg()
    o.reduce_ajdg()
    assert rel_l2(g.download_field("aj"), o.f["aj"]) < TOL
    assert rel_l2(g.download_field("ajdg"), o.f["ajdg"]) < TOL


@pytest.mark.parametrize("func", [0, 1, 2])
def test_charge_routing(gpu, func):
    c = case()
    cfg, eb, p, tp = build(c)
    p["preside"][::7] = -1
    p["preside"][3::11] = -2
    p["nid"][5::13] = -1
    g = Emses(cfg)
    g.upload_particles(p, tp)
    o = O.Oracle(cfg, p, tp, eb)
    g.charge(1, func)
    o.charge(func)
    pg, _ = g.download_particles()
    assert same_particles(pg, o.pbuf)
    for name in ("rho", "rhodg", "rhobk", "rhobksp"):
        assert rel_l2(g.download_field(name), o.f[name]) < TOL, name
    for name in ("rho", "rhobk", "rhobksp"):
        g.reduce_rho(name)
        o.reduce_rho(name)
        assert rel_l2(g.download_field(name), o.f[name]) < TOL, name


@pytest.mark.parametrize("nfbnd", [(0, 0, 0), (0, 0, 1), (1, 1, 1), (2, 0, 2)])
def test_guard_folds_bit_exact(gpu, nfbnd):
    c = case(n=(6, 7, 8), nfbnd=nfbnd)
    cfg, eb, p, tp = build(c)
    rng = np.random.default_rng(9)
    g = Emses(cfg)
    o = O.Oracle(cfg, p, tp, eb)
    for name in ("rho", "aj", "ajdg", "rhodg"):
        raw = rng.normal(size=o.f[name].shape)
        o.f[name][...] = raw
        g.upload_field(name, raw)
    g.reduce_rho("rho"); o.reduce_rho("rho")
    g.reduce_rho("rhodg"); o.reduce_rho("rhodg")
    g.reduce_aj(); o.reduce_aj()
    g.reduce_ajdg(); o.reduce_ajdg()
    for name in ("rho", "rhodg", "aj", "ajdg"):
        assert np.array_equal(g.download_field(name), o.f[name]), name


def test_rhoupd_and_energy(gpu):
    c = case()
    cfg, g, o = pair(c)
    rng = np.random.default_rng(4)
    for name in ("rho", "aj"):
        raw = rng.normal(size=o.f[name].shape)
        o.f[name][...] = raw
        g.upload_field(name, raw)
    g.rhoupd(1)
    o.rhoupd()
    assert np.array_equal(g.download_field("rho"), o.f["rho"])
    e = g.energy()
    assert np.allclose(e, o.energy(), rtol=TOL, atol=0)


@pytest.mark.parametrize("tile", [(0, 0, 0), (4, 4, 4), (3, 5, 2)])
def test_spsort_permutation_exact(gpu, tile):
    c = case(n=(9, 10, 8), tile=tile)
    cfg, eb, p, tp = build(c)
    rng = np.random.default_rng(1)
    perm = np.concatenate([rng.permutation(tp[0]), tp[0] + rng.permutation(tp[1])])
    p = p[perm]
    p["pid"] = np.arange(p.size) % 15
    g = Emses(cfg)
    g.upload_particles(p, tp)
    o = O.Oracle(cfg, p, tp, eb)
    g.spsort(1)
    o.spsort()
    pg, _ = g.download_particles()
    assert same_particles(pg, o.pbuf)


def test_spsort_large_multi_block(gpu):
    """~1M particles: many radix blocks and a two-level prefix sum."""
    c = case(n=(64, 64, 64), ppc=(2, 2), tile=(8, 8, 8))
    cfg, eb, p, tp = build(c)
    rng = np.random.default_rng(2)
    perm = np.concatenate([rng.permutation(tp[0]), tp[0] + rng.permutation(tp[1])])
    p = p[perm]
    g = Emses(cfg)
    g.upload_particles(p, tp)
    o = O.Oracle(cfg, p, tp, eb)
    g.spsort(1)
    o.spsort()
    pg, _ = g.download_particles()
    assert same_particles(pg, o.pbuf)
    p["nid"][::3] = -1
    g.upload_particles(p, tp)
    o = O.Oracle(cfg, p, tp, eb)
    assert np.array_equal(g.compact(1), (o.compact(), o.totalp)[1])
    pg, _ = g.download_particles()
    assert same_particles(pg, o.pbuf)


def test_compact_exact(gpu):
    c = case()
    cfg, eb, p, tp = build(c)
    p["nid"][::5] = -1
    p["nid"][tp[0]:][::3] = -1
    g = Emses(cfg)
    g.upload_particles(p, tp)
    o = O.Oracle(cfg, p, tp, eb)
    tpg = g.compact(1)
    o.compact()
    assert np.array_equal(tpg, o.totalp)
    pg, _ = g.download_particles()
    assert same_particles(pg, o.pbuf)


def test_injected_particles_hash_stream(gpu):
    c = case()
    cfg, eb, p, tp = build(c)
    p["preside"][::9] = 1
    g = Emses(cfg)
    g.upload_particles(p, tp)
    g.upload_field("eb", eb)
    o = O.Oracle(cfg, p, tp, eb)
    g.grdcrt(1); o.grdcrt()
    for _ in range(2):
        g.psolve2(1, 2)
        o.psolve2(2)
    pg, _ = g.download_particles()
    assert same_particles(pg, o.pbuf)


def test_injected_particles_ranu0_stream(gpu):
    """rng_mode 1 with the reference's own RANU0 stream (MT19937 of
    lib/mtarm, compiled in oracle/_ref) gives the reference's fractions."""
    if O.ref_lib() is None:
        pytest.skip("oracle/_ref not built")
    c = case()
    cfg, eb, p, tp = build(c)
    cfg.rng_mode = 1
    p["preside"][1::6] = 1
    u = O.ranu0_stream(10, int((p["preside"] == 1).sum()) * 2)
    g = Emses(cfg)
    g.upload_particles(p, tp)
    g.upload_field("eb", eb)
    g.set_randoms(u)
    o = O.Oracle(cfg, p, tp, eb)
    o.set_randoms(u)
    g.grdcrt(1); o.grdcrt()
    g.zero_field("aj")
    g.psolve1(1, 2, 0)
    o.psolve1(2, 0)
    pg, _ = g.download_particles()
    assert same_particles(pg, o.pbuf)
    assert rel_l2(g.download_field("aj"), o.f["aj"]) < TOL


def test_ten_step_run_stays_bit_exact(gpu):
    """Config-1 physics (scaled to 12^3 x 8 ppc) for 10 steps of grdcrt ->
    psolve2 -> compact -> spsort every 4 -> charge -> reduce."""
    c = case(n=(12, 12, 12), ppc=(8, 8), tile=(4, 4, 4))
    cfg, g, o = pair(c)
    for step in range(1, 11):
        g.grdcrt(1); o.grdcrt()
        g.psolve2(1, 2); o.psolve2(2)
        g.compact(1); o.compact()
        if step % 4 == 0:
            g.spsort(1); o.spsort()
        g.charge(1, 0); o.charge(0)
        g.reduce_rho("rho"); o.reduce_rho("rho")
    pg, tpg = g.download_particles()
    assert np.array_equal(tpg, o.totalp)
    assert same_particles(pg, o.pbuf)
    assert rel_l2(g.download_field("rho"), o.f["rho"]) < TOL


def test_ps2_is_unsupported(gpu):
    from ctca_b200.emses import ERR_UNSUPPORTED, EmsesError
    cfg, g, o = pair(case())
    with pytest.raises(EmsesError) as e:
        g.grdcrt(2)
    assert e.value.code == ERR_UNSUPPORTED
