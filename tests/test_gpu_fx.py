"""Parity of the FP32 / fixed-point form with the FP64 oracle.

The FP32 form starts from the FP32-rounded state (fx_load -> fx_store), the
oracle runs psolve1 + add_boundary_current and charge + add_boundary_charge
on that same state for one step, and the outputs agree within:
  rho, J : L2 relative error <= 1e-5 (the stated tolerance of the form)
  positions / velocities : max abs error <= 1e-5 (cells) / 1e-5 relative
  cell indices : exact, except particles within 1e-5 of a cell face.
The fixed-point sums are bit-reproducible: two runs give identical int64
accumulators."""
import numpy as np
import pytest

from ctca_b200.emses import FX_ROW_SLOTS, Emses
from oracle import oracle as O

from helpers import build, case, rel_l2

pytestmark = pytest.mark.gpu

RHOJ_TOL = 1e-5


def fx_pair(c, capacity_factor=1.0):
    cfg, eb, p, tp = build(c, capacity_factor)
    g = Emses(cfg)
    g.upload_particles(p, tp)
    g.upload_field("eb", eb)
    g.fx_load()
    g.fx_store()           # FP32-rounded, tile-sorted state as FP64 records
    p32, tp32 = g.download_particles()
    g.fx_load()
    o = O.Oracle(cfg, p32, tp32, eb)
    return cfg, g, o, p32, tp32


def oracle_step(o, ustep=2):
    o.grdcrt()
    o.f["aj"][...] = 0.0
    o.psolve1(ustep, 0)
    o.reduce_aj()
    o.charge(0)
    o.reduce_rho("rho")


def near_face(x, eps=1e-5):
    f = x - np.floor(x)
    return (f < eps) | (f > 1 - eps)


@pytest.mark.parametrize("npbnd,nfbnd", [((0, 0, 0), (0, 0, 0)), ((1, 1, 1), (1, 1, 1)), ((0, 0, 2), (0, 0, 1))])
def test_fx_one_step_vs_oracle(gpu, npbnd, nfbnd):
    c = case(n=(16, 16, 16), ppc=(8, 8), npbnd=npbnd, nfbnd=nfbnd, vth_scale=3.0, tile=(8, 8, 8))
    cfg, g, o, p32, tp32 = fx_pair(c)
    g.fx_step(2, False)
    oracle_step(o)
    rho_err = rel_l2(g.download_field("rho"), o.f["rho"])
    aj_err = rel_l2(g.download_field("aj"), o.f["aj"])
    print(f"rho L2 rel {rho_err:.3e}  J L2 rel {aj_err:.3e}")
    assert rho_err < RHOJ_TOL
    assert aj_err < RHOJ_TOL
    g.fx_store()  # same buffer order as the oracle's pbuf; dead ones in place
    pg, tpg = g.download_particles()
    assert np.array_equal(tpg, o.totalp)
    assert np.array_equal(pg["nid"], o.pbuf["nid"])
    a, b = pg[o.pbuf["nid"] != -1], o.pbuf[o.pbuf["nid"] != -1]
    vmax = max(np.max(np.abs(b["vx"])), np.max(np.abs(b["vy"])), np.max(np.abs(b["vz"])))
    for f in ("vx", "vy", "vz"):
        err = np.max(np.abs(a[f] - b[f])) / vmax
        print(f"{f} max rel {err:.2e}")
        assert err <= 1e-5
    for f, n in (("x", cfg.nx), ("y", cfg.ny), ("z", cfg.nz)):
        d = np.abs(a[f] - b[f])
        d = np.minimum(d, np.abs(d - n))  # periodic wrap
        print(f"{f} max abs {np.max(d):.2e}")
        assert np.max(d) < 1e-5
        ok = ~near_face(b[f])
        assert np.array_equal(np.floor(a[f][ok]), np.floor(b[f][ok]))


def test_fx_is_bit_reproducible(gpu):
    c = case(n=(16, 16, 16), ppc=(8, 8), tile=(8, 8, 8))
    cfg, eb, p, tp = build(c)
    accs = []
    for _ in range(2):
        g = Emses(cfg)
        g.upload_particles(p, tp)
        g.upload_field("eb", eb)
        g.fx_load()
        g.fx_step(2, False)
        g.fx_step(2, True)
        accs.append(g.fx_download_accum())
        g.close()
    assert np.array_equal(accs[0][0], accs[1][0])
    assert np.array_equal(accs[0][1], accs[1][1])


def test_fx_sort_matches_oracle_keys(gpu):
    c = case(n=(16, 8, 24), ppc=(5, 3), tile=(8, 4, 8))
    cfg, g, o, p32, tp32 = fx_pair(c)
    # fx_store output is tile-sorted: same order as the oracle's stable sort
    o.spsort()
    from helpers import same_particles
    assert same_particles(p32, o.pbuf)


def test_fx_multi_step_tracks_oracle(gpu):
    """Four steps with a sort in between: rho/J stay within tolerance of the
    oracle run from the same FP32-rounded start."""
    c = case(n=(16, 16, 16), ppc=(8, 8), tile=(8, 8, 8))
    cfg, g, o, p32, tp32 = fx_pair(c)
    for step in range(4):
        g.fx_step(2, step == 2)
        if step == 2:
            o.spsort()
        oracle_step(o)
    assert rel_l2(g.download_field("rho"), o.f["rho"]) < RHOJ_TOL
    assert rel_l2(g.download_field("aj"), o.f["aj"]) < RHOJ_TOL
    assert np.array_equal(g.fx_counts(), o.totalp)


def test_fx_escape_counts(gpu):
    c = case(n=(16, 16, 16), ppc=(8, 8), npbnd=(2, 2, 2), nfbnd=(1, 1, 1), vth_scale=6.0, tile=(8, 8, 8))
    cfg, g, o, p32, tp32 = fx_pair(c)
    for _ in range(3):
        g.fx_step(2, False)
        oracle_step(o)
    g.fx_sort()
    assert np.array_equal(g.fx_counts(), [(o.pbuf[:o.totalp[0]]["nid"] != -1).sum(),
                                          (o.pbuf[o.totalp[0]:]["nid"] != -1).sum()])


def _tile_key(cfg, tile, p):
    i, j, k = np.floor(p["x"]).astype(int), np.floor(p["y"]).astype(int), np.floor(p["z"]).astype(int)
    nt = [-(-n // t) for n, t in zip((cfg.nx, cfg.ny, cfg.nz), tile)]
    tid = i // tile[0] + nt[0] * (j // tile[1] + nt[1] * (k // tile[2]))
    lin = i % tile[0] + tile[0] * (j % tile[1] + tile[1] * (k % tile[2]))
    return tid * (tile[0] * tile[1] * tile[2]) + lin, tid


@pytest.mark.parametrize("npbnd,tile,ppc,n", [
    ((0, 0, 0), (8, 8, 8), (8, 8), (16, 16, 16)),
    ((1, 2, 0), (8, 4, 8), (8, 8), (16, 16, 16)),
    # tiles of 28 rows: the move's small shape, 40-column windows; of 1
    # row: one group of the whole row
    ((0, 0, 0), (8, 8, 8), (40, 1), (16, 16, 16)),
    # tiles of 45 rows: the mid shape, three buffers
    ((0, 0, 0), (8, 8, 8), (64, 4), (16, 16, 16)),
    # tiles of 67 rows: the large shape with windows
    ((0, 0, 0), (8, 8, 8), (96, 4), (16, 16, 16)),
    # tiles of 98 rows: no window, inv read from global memory, several
    # batches of slots per group
    ((0, 0, 0), (8, 8, 8), (140, 4), (16, 16, 16)),
    # partial tiles: grid sizes that are not multiples of the tile, periodic
    # (the last tile's sort box wraps onto the first tile) and not
    ((0, 0, 0), (8, 8, 8), (8, 8), (20, 12, 18)),
    ((1, 2, 0), (8, 8, 8), (8, 8), (13, 22, 9)),
])
def test_fx_local_sort_is_a_stable_cell_sort(gpu, npbnd, tile, ppc, n):
    """The re-sort after a step (the tile-local counting sort) orders the
    live particles by the tile-major cell key; equal cells keep the order
    (source tile, warp, row, lane) of the thread-major layout of the last
    sort, computed here from the tile sizes of that sort."""
    threads = FX_ROW_SLOTS
    c = case(n=n, ppc=ppc, npbnd=npbnd, vth_scale=6.0, tile=tile)
    cfg, eb, p, tp = build(c)
    g = Emses(cfg)
    g.upload_particles(p, tp)
    g.upload_field("eb", eb)
    g.fx_load()
    g.fx_store()
    p0, tp0 = g.download_particles()   # sorted; cells of the last sort
    g.fx_step(2, False)
    g.fx_store()
    p1, tp1 = g.download_particles()   # same order, moved
    g.fx_sort()
    g.fx_store()
    p2, tp2 = g.download_particles()
    base0 = np.concatenate([[0], np.cumsum(tp0)])
    for s in range(cfg.nspec):
        a0 = p0[base0[s]:base0[s] + tp0[s]]
        a1 = p1[base0[s]:base0[s] + tp0[s]]
        _, t0 = _tile_key(cfg, tile, a0)
        ntile = int(t0.max()) + 1
        counts = np.bincount(t0, minlength=ntile)
        starts = np.concatenate([[0], np.cumsum(counts)])
        q = np.arange(a0.size) - starts[t0]
        L = -(-counts[t0] // threads)
        col, row = q // L, q % L
        src = np.lexsort((col % 32, row, col // 32, t0))  # (tile, warp, row, lane)
        order_pos = np.empty(a0.size, dtype=np.int64)
        order_pos[src] = np.arange(a0.size)
        live = a1["nid"] != -1
        key1, _ = _tile_key(cfg, tile, a1)
        idx = np.flatnonzero(live)
        exp = idx[np.lexsort((order_pos[idx], key1[idx]))]
        base2 = int(np.sum(tp2[:s]))
        got = p2[base2:base2 + tp2[s]]
        assert tp2[s] == live.sum()
        for f in ("x", "y", "z", "vx", "vy", "vz"):
            assert np.array_equal(got[f], a1[exp][f]), (s, f)
    g.close()


def test_fx_em_step_vs_oracle(gpu):
    """One EM step with the fields on the device (bfield, push, J, bfield,
    efield, border exchange) against the oracle's FP64 sequence on the same
    FP32-rounded start: the fields agree to the FP32 form's J tolerance."""
    c = case(n=(16, 16, 16), ppc=(8, 8), vth_scale=3.0, tile=(8, 8, 8))
    cfg, g, o, p32, tp32 = fx_pair(c)
    tcs = 0.125
    g.fx_em_step(2, False, tcs)
    o.bfield()
    oracle_step(o)
    o.bfield()
    o.efield(tcs)
    o.exchange_eb()
    eb = g.download_field("eb")
    err = rel_l2(eb, o.eb)
    print(f"eb L2 rel {err:.3e}")
    assert err < 1e-6
    assert rel_l2(g.download_field("aj"), o.f["aj"]) < RHOJ_TOL
    g.close()


def test_fx_empty_species_tracks_oracle(gpu):
    """A species without particles: steps and sorts (tile-local) leave it
    empty and the other species tracks the oracle."""
    c = case(n=(16, 16, 16), ppc=(8, 0), tile=(8, 8, 8))
    cfg, g, o, p32, tp32 = fx_pair(c)
    assert tp32[1] == 0
    for step in range(4):
        g.fx_step(2, step == 1)
        if step == 1:
            o.spsort()
        oracle_step(o)
    assert rel_l2(g.download_field("rho"), o.f["rho"]) < RHOJ_TOL
    assert rel_l2(g.download_field("aj"), o.f["aj"]) < RHOJ_TOL
    assert np.array_equal(g.fx_counts(), o.totalp)
    g.close()


def test_fx_stray_particles_fall_back_to_the_radix_sort(gpu):
    """Particles that left their tile's sort box (tile + one cell) between
    sorts: the tile-local sort gives way to the radix sort, which keeps every
    live particle and orders them by the tile-major cell key; the next step
    still tracks the oracle."""
    tile = (8, 8, 8)
    c = case(n=(16, 16, 16), ppc=(4, 4), vth_scale=20.0, tile=tile)
    cfg, g, o, p32, tp32 = fx_pair(c)
    for _ in range(3):
        g.fx_step(2, False)
        oracle_step(o)
    g.fx_store()
    pa, ta = g.download_particles()     # slot order of the load: same as p32
    # some particle is out of the sort box of the tile it was sorted into
    ext = np.array([cfg.nx, cfg.ny, cfg.nz])
    c0 = np.stack([np.floor(p32[f]) for f in "xyz"], 1).astype(int)
    c1 = np.stack([np.floor(pa[f]) for f in "xyz"], 1).astype(int)
    lo = (c0 // tile) * tile - 1
    off = (c1 - lo) % ext              # periodic
    stray = (pa["nid"] != -1) & np.any(off >= np.array(tile) + 2, axis=1)
    assert stray.sum() > 0
    g.fx_sort()
    g.fx_store()
    pb, tb = g.download_particles()
    fields = ("x", "y", "z", "vx", "vy", "vz")
    base_a = np.concatenate([[0], np.cumsum(ta)])
    base_b = np.concatenate([[0], np.cumsum(tb)])
    for s in range(cfg.nspec):
        a = pa[base_a[s]:base_a[s + 1]]
        a = a[a["nid"] != -1]
        b = pb[base_b[s]:base_b[s + 1]]
        assert b.size == a.size
        key, _ = _tile_key(cfg, tile, b)
        assert np.all(np.diff(key) >= 0)
        ka = np.lexsort([a[f] for f in fields])
        kb = np.lexsort([b[f] for f in fields])
        for f in fields:
            assert np.array_equal(a[f][ka], b[f][kb]), (s, f)
    g.fx_step(2, False)
    o.spsort()
    oracle_step(o)
    assert rel_l2(g.download_field("rho"), o.f["rho"]) < RHOJ_TOL
    assert rel_l2(g.download_field("aj"), o.f["aj"]) < RHOJ_TOL
    g.close()


def test_step_download_overlap_matches_plain_io(gpu):
    """emsesg_fx_step_download with the next eb uploaded asynchronously (a
    different eb every step, so that the double buffer must hand over the
    right one; copied in z chunks, the push in two parts) gives the rho / aj
    and the particles of the plain sequence upload_field, fx_step,
    download_field through sorts: the first step (the eb already there, one
    launch) bit for bit, the others up to the last-bit rounding of the
    particles the parts deferred."""
    import torch
    c = case(n=(16, 16, 16), ppc=(8, 8), vth_scale=2.0, tile=(8, 8, 8))
    cfg, eb, p, tp = build(c, 1.2)
    ebs = [np.ascontiguousarray(eb * (1.0 + 0.05 * k)) for k in range(6)]
    pinned = [torch.from_numpy(e.reshape(-1)).pin_memory().numpy() for e in ebs]
    with Emses(cfg) as a, Emses(cfg) as b:
        for g in (a, b):
            g.upload_particles(p, tp)
            g.upload_field("eb", ebs[0])
            g.fx_load()
        rho_b = torch.empty(b.field_size("rho"), dtype=torch.float64).pin_memory().numpy()
        aj_b = torch.empty(b.field_size("aj"), dtype=torch.float64).pin_memory().numpy()
        for k in range(6):
            srt = k % 3 == 2
            a.upload_field("eb", ebs[k])
            a.fx_step(2, srt)
            ra, ja = a.download_field("rho"), a.download_field("aj")
            if k > 0:
                b.upload_eb_async(pinned[k])
            b.fx_step_download(2, srt, rho_b, aj_b)
            if k == 0:
                assert np.array_equal(ra.reshape(-1), rho_b) and np.array_equal(ja.reshape(-1), aj_b)
            a.fx_store()
            b.fx_store()
            pa, ta = a.download_particles()
            pb, tb = b.download_particles()
            assert np.array_equal(ta, tb)
            assert_same_up_to_deferred(pa, pb, ra.reshape(-1), rho_b, ja.reshape(-1), aj_b)


def assert_same_up_to_deferred(pa, pb, ra, rb, ja, jb):
    """The state of a step pushed in parts against the same step pushed in
    one launch: the particles the parts deferred (k_fx_deferred) may round
    their kick otherwise in the last bit, so positions agree to 1e-5 cell,
    velocities to 1e-6 of the largest, rho and J to 1e-7 relative L2; the
    rest, and every particle's cell and liveness, bit for bit."""
    assert np.array_equal(pa["nid"], pb["nid"])
    for f in ("x", "y", "z"):
        assert np.array_equal(np.floor(pa[f]), np.floor(pb[f])), f
        assert np.max(np.abs(pa[f] - pb[f]), initial=0.0) < 1e-5, f
    vmax = max(np.abs(pa[f]).max() for f in ("vx", "vy", "vz"))
    for f in ("vx", "vy", "vz"):
        assert np.max(np.abs(pa[f] - pb[f]), initial=0.0) < 1e-6 * vmax, f
    differ = ~np.all(pa.view(np.uint8).reshape(pa.size, -1) == pb.view(np.uint8).reshape(pb.size, -1), axis=1)
    assert differ.sum() <= max(4, pa.size // 1000)
    assert rel_l2(ra, rb) < 1e-7 and rel_l2(ja, jb) < 1e-7


@pytest.mark.parametrize("es,bodies", [(False, False), (True, False), (False, True)])
def test_eb_in_z_chunks_matches_one_launch(gpu, es, bodies):
    """An asynchronous eb upload arrives in z chunks and the push runs in
    parts, each once its chunk is there (four tile layers: four parts); a
    particle outside its tile's box whose node planes are not there yet
    (those of the low layers that crossed the periodic z face since the
    sort gather from the top planes) is pushed after the last part.  The
    counters equal those of the step after a synchronous upload, every step,
    with and without the current, with a box body (absorption, and loaded
    particles inside it on the general path of the first step), through
    re-sorts, a different eb every step; particles, rho and J agree up to
    the last-bit rounding of the deferred particles."""
    import torch
    c = case(n=(16, 12, 32), ppc=(8, 8), vth_scale=6.0, tile=(8, 4, 8))
    if bodies:
        c.bodies = [dict(geotype=0, ncond=1, xlpc=4.0, xupc=9.0, ylpc=3.0, yupc=8.0, zlpc=2.0, zupc=7.0,
                         sqdscaled=1.0)]
    cfg, eb, p, tp = build(c, 1.2)
    rng = np.random.default_rng(17)
    ebs = [np.ascontiguousarray(eb + 0.02 * k * rng.standard_normal(eb.shape)) for k in range(7)]
    pinned = [torch.from_numpy(e.reshape(-1)).pin_memory().numpy() for e in ebs]
    with Emses(cfg) as a, Emses(cfg) as b:
        for g in (a, b):
            g.upload_particles(p, tp)
            g.upload_field("eb", ebs[0])
            g.fx_load()
        for k in range(7):
            srt = k % 4 == 3
            a.upload_field("eb", ebs[k])
            b.upload_eb_async(pinned[k])
            for g in (a, b):
                (g.fx_step_es if es else g.fx_step)(2, srt)
            ca, cb = a.get_counters().as_dict(), b.get_counters().as_dict()
            for key in ca:
                assert np.array_equal(ca[key], cb[key]), (k, key)
            for g in (a, b):
                g.fx_store()
            pa, ta = a.download_particles()
            pb, tb = b.download_particles()
            assert np.array_equal(ta, tb)
            assert_same_up_to_deferred(pa, pb, a.download_field("rho"), b.download_field("rho"),
                                       a.download_field("aj"), b.download_field("aj"))
        if bodies:
            assert ca["influx"].sum() > 0


def test_async_eb_upload_with_graph_runs(gpu):
    """An asynchronous eb upload between graph runs (emsesg_fx_run) takes
    effect at the next run, whose graph is captured again for the other eb
    buffer: the same particles and rho / aj, bit for bit, as synchronous
    uploads and step-by-step runs; a batch refuses to launch after an
    asynchronous upload of one of its runs."""
    import torch
    from ctca_b200.emses import Batch, EmsesError
    c = case(n=(16, 16, 16), ppc=(6, 6), vth_scale=2.0, tile=(8, 8, 8))
    cfg, eb, p, tp = build(c, 1.2)
    ebs = [np.ascontiguousarray(eb * (1.0 + 0.07 * k)) for k in range(3)]
    pinned = [torch.from_numpy(e.reshape(-1)).pin_memory().numpy() for e in ebs]
    with Emses(cfg) as a, Emses(cfg) as b:
        for g in (a, b):
            g.upload_particles(p, tp)
            g.upload_field("eb", ebs[0])
            g.fx_load()
        for k in range(3):
            if k > 0:
                a.upload_field("eb", ebs[k])
                b.upload_eb_async(pinned[k])
            a.fx_run(2, 8, 4, use_graph=False)
            b.fx_run(2, 8, 4, use_graph=True)
            a.synchronize()
            b.synchronize()
            assert np.array_equal(a.download_field("rho"), b.download_field("rho")), k
            assert np.array_equal(a.download_field("aj"), b.download_field("aj")), k
        a.fx_store()
        b.fx_store()
        pa, _ = a.download_particles()
        pb, _ = b.download_particles()
        assert np.array_equal(pa.view(np.uint8), pb.view(np.uint8))
        b.fx_load()
        batch = Batch([b], 2, 8, [4])
        batch.launch(1)
        b.synchronize()
        b.upload_eb_async(pinned[0])
        with pytest.raises(EmsesError, match="asynchronously"):
            batch.launch(1)
        batch.close()


@pytest.mark.parametrize("npbnd,nfbnd,bodies,tile", [((0, 0, 0), (0, 0, 0), False, (8, 8, 8)),
                                                     ((0, 0, 2), (0, 0, 1), True, (8, 8, 8)),
                                                     ((1, 0, 2), (1, 0, 1), True, (4, 4, 4))])
def test_es_step_is_the_step_without_current(gpu, npbnd, nfbnd, bodies, tile):
    """emsesg_fx_step_es (psolve2 + charge on the FP32 form): the same
    particles, counts and rho, bit for bit, as emsesg_fx_step from the same
    state, over steps with re-sorts, escapes, injected particles (inflow
    through the open z face, their first push on the tail path) and (with
    bodies) absorption by a box, a cylinder and a sphere; aj is left as it
    was.  Against the oracle's psolve2 + charge from the same state: rho
    within 1e-5."""
    c = case(n=(16, 16, 24), ppc=(8, 8), npbnd=npbnd, nfbnd=nfbnd, vth_scale=3.0, tile=tile)
    if bodies:
        c.bodies = [dict(geotype=0, ncond=1, xlpc=3.0, xupc=7.0, ylpc=3.0, yupc=7.0, zlpc=4.0, zupc=9.0,
                         sqdscaled=1.0),
                    dict(geotype=2, ncond=1, cyl_align=3, cyl_axis=(11.5, 11.25), cyl_edge=(2.0, 20.0), radius=2.2,
                         sqdscaled=1.0),
                    dict(geotype=3, ncond=0, sph_center=(5.3, 11.7, 16.1), radius=2.4)]
    cfg, eb, p, tp = build(c, 1.2)
    with Emses(cfg) as a, Emses(cfg) as b:
        for g in (a, b):
            g.upload_particles(p, tp)
            g.upload_field("eb", eb)
            g.fx_load()
        aj0 = b.download_field("aj")
        if npbnd[2] == 2:
            # inflow through the back z face before every step (the tail
            # zone's first push, with the random fractions of the step)
            from ctca_b200 import inject
            rng = np.random.default_rng(12)
            vz = np.sort(rng.uniform(-0.2, -0.01, 256))
            vxy = rng.normal(0.0, 0.05, 256)
            uni = rng.random(100000)
            for g in (a, b):
                g.set_randoms(uni)
        for k in range(5):
            srt = k % 2 == 1
            if npbnd[2] == 2 and k != 2:  # (step 2 is the one compared with the oracle)
                for s in (1, 2):
                    rec = inject.inflow_z(False, 50, cfg.nx, cfg.ny, cfg.nz, vz, vxy, vxy, 1.0,
                                          np.random.default_rng(100 * k + s), spec=s)
                    a.fx_inject(s, rec)
                    b.fx_inject(s, rec)
            if k == 2:
                # the oracle from the ES step's state: psolve2 + charge
                b.fx_store()
                pb, tpb = b.download_particles()
                b.fx_load()
                a.fx_store()
                a.fx_load()
                o = O.Oracle(cfg, pb, tpb, eb)
                o.grdcrt()
                o.psolve2(2)
                o.charge(0)
                o.reduce_rho("rho")
            a.fx_step(2, srt)
            b.fx_step_es(2, srt)
            assert np.array_equal(a.download_field("rho"), b.download_field("rho")), k
            assert np.array_equal(a.fx_counts(), b.fx_counts()), k
            if k == 2:
                err = rel_l2(b.download_field("rho"), o.f["rho"])
                print(f"rho against psolve2 + charge: {err:.2e}")
                assert err < RHOJ_TOL
        assert np.array_equal(b.download_field("aj"), aj0)
        ca, cb = a.get_counters().as_dict(), b.get_counters().as_dict()
        assert np.array_equal(ca["influx"], cb["influx"]) and np.array_equal(ca["nesc"], cb["nesc"])
        if bodies:
            assert int(cb["influx"][:2].sum()) > 0
        a.fx_store()
        b.fx_store()
        pa, _ = a.download_particles()
        pb, _ = b.download_particles()
        assert np.array_equal(pa.view(np.uint8), pb.view(np.uint8))


def test_es_entry_points_refuse_bad_arguments(gpu):
    """The electrostatic entry points: a Poisson boundary other than 0, 1, 2
    and mltstp < 1 are argument errors; the step without the current is
    refused in slab mode; the context stays usable after each refusal."""
    from ctca_b200.emses import ERR_ARG, ERR_STATE, EmsesError
    c = case(n=(16, 16, 16), ppc=(2, 2), tile=(8, 8, 8))
    cfg, eb, p, tp = build(c, 1.2)
    with Emses(cfg) as g:
        g.upload_particles(p, tp)
        g.upload_field("eb", eb)
        g.fx_load()
        with pytest.raises(EmsesError) as e:
            g.esfield(1, mtd_vbnd=(0, 3, 0))
        assert e.value.code == ERR_ARG
        with pytest.raises(EmsesError) as e:
            g.esfield(0)
        assert e.value.code == ERR_ARG
        g.fx_step_es(2, False)
        assert g.esfield(1) >= 0.0
        g.fx_slab(True, 1000)
        with pytest.raises(EmsesError) as e:
            g.fx_step_es(2, False)
        assert e.value.code == ERR_STATE


@pytest.mark.parametrize("ustep", [1, 4])
def test_fx_one_step_other_usteps(gpu, ustep):
    """The push with ustep other than 2 (the time step in units of dth: the
    kick E * qm * ustep / 2, the move v * ustep, the current (a - b) / ustep)
    against the oracle's psolve1 + charge from the same state."""
    c = case(n=(16, 16, 16), ppc=(8, 8), npbnd=(0, 0, 0), nfbnd=(0, 0, 0), vth_scale=2.0, tile=(8, 8, 8))
    cfg, g, o, p32, tp32 = fx_pair(c)
    g.fx_step(ustep, False)
    oracle_step(o, ustep)
    rho_err = rel_l2(g.download_field("rho"), o.f["rho"])
    aj_err = rel_l2(g.download_field("aj"), o.f["aj"])
    print(f"ustep {ustep}: rho {rho_err:.2e}, J {aj_err:.2e}")
    assert rho_err < RHOJ_TOL and aj_err < RHOJ_TOL
    g.close()


def test_fx_species_with_their_own_boundaries(gpu):
    """npbnd per species (electrons periodic in x and escaping in z, ions
    reflecting in x and periodic in z): two steps with a re-sort against
    the oracle started from the FP32 state before each."""
    c = case(n=(16, 16, 16), ppc=(8, 8), nfbnd=(0, 0, 1), vth_scale=3.0, tile=(8, 8, 8))
    c.species[0].npbnd = (0, 0, 2)
    c.species[1].npbnd = (1, 0, 0)
    cfg, g, o, p32, tp32 = fx_pair(c, 1.2)
    for k in range(2):
        if k:
            g.fx_store()
            p32, tp32 = g.download_particles()
            g.fx_load()
            o = O.Oracle(cfg, p32, tp32, o.eb)
        g.fx_step(2, k == 0)
        oracle_step(o)
        rho_err = rel_l2(g.download_field("rho"), o.f["rho"])
        aj_err = rel_l2(g.download_field("aj"), o.f["aj"])
        print(f"step {k}: rho {rho_err:.2e}, J {aj_err:.2e}")
        assert rho_err < RHOJ_TOL and aj_err < RHOJ_TOL
    nesc = g.get_counters().as_dict()["nesc"]
    assert nesc[0] > 0 and nesc[1] == 0
    g.close()


@pytest.mark.parametrize("nspec", [1, 3])
def test_fx_other_species_counts(gpu, nspec):
    """One species (electrons alone) and three (a second, heavier ion
    population with its own density): two steps with a re-sort against the
    oracle, with and without the current -- the per-species regions, launch
    rows and counters of the FP32 form for species counts other than two."""
    from ctca_b200.inputs import Species
    c = case(n=(16, 16, 16), ppc=(8, 8), vth_scale=2.0, tile=(8, 8, 8))
    if nspec == 1:
        c.species = c.species[:1]
    else:
        c.species.append(Species(ppc=4, qm=1.0 / 400.0, vth=c.species[1].vth * 0.5, drift=(0.0, 0.01, 0.0)))
    cfg, g, o, p32, tp32 = fx_pair(c, 1.2)
    assert cfg.nspec == nspec
    for k in range(3):
        if k:
            g.fx_store()
            p32, tp32 = g.download_particles()
            g.fx_load()
            o = O.Oracle(cfg, p32, tp32, o.eb)
        es = k == 2
        if es:
            g.fx_step_es(2, False)
            o.grdcrt()
            o.psolve2(2)
            o.charge(0)
            o.reduce_rho("rho")
        else:
            g.fx_step(2, k == 0)
            oracle_step(o)
        rho_err = rel_l2(g.download_field("rho"), o.f["rho"])
        msg = f"nspec {nspec} step {k}: rho {rho_err:.2e}"
        assert rho_err < RHOJ_TOL, msg
        if not es:
            aj_err = rel_l2(g.download_field("aj"), o.f["aj"])
            msg += f", J {aj_err:.2e}"
            assert aj_err < RHOJ_TOL, msg
        print(msg)
        assert np.array_equal(g.fx_counts(), o.totalp[:nspec]), k
    e = g.fx_energy()
    assert e.shape[0] == nspec and np.all(e > 0)
    g.close()


@pytest.mark.parametrize("n,npbnd,nfbnd", [((20, 12, 18), (0, 0, 0), (0, 0, 0)), ((13, 22, 9), (1, 0, 2), (1, 0, 1))])
def test_fx_partial_tiles(gpu, n, npbnd, nfbnd):
    """Grid sizes that are not multiples of the 8-cell sort tile (partial
    tiles on every axis, odd sizes): steps with re-sorts against the oracle,
    and the tile-local sort's order against its definition."""
    c = case(n=n, ppc=(6, 6), npbnd=npbnd, nfbnd=nfbnd, vth_scale=3.0, tile=(8, 8, 8))
    cfg, g, o, p32, tp32 = fx_pair(c, 1.2)
    for k in range(3):
        if k:
            g.fx_store()
            p32, tp32 = g.download_particles()
            g.fx_load()
            o = O.Oracle(cfg, p32, tp32, o.eb)
        g.fx_step(2, k == 1)
        oracle_step(o)
        rho_err = rel_l2(g.download_field("rho"), o.f["rho"])
        aj_err = rel_l2(g.download_field("aj"), o.f["aj"])
        print(f"{n} step {k}: rho {rho_err:.2e}, J {aj_err:.2e}")
        assert rho_err < RHOJ_TOL and aj_err < RHOJ_TOL
        # live particles per species (the re-sort drops the dead ones; the
        # oracle keeps them in place until a compaction)
        base = np.concatenate([[0], np.cumsum(o.totalp[:cfg.nspec])])
        live = [int((o.pbuf["nid"][base[s]:base[s + 1]] != -1).sum()) for s in range(cfg.nspec)]
        if k == 1:
            assert list(g.fx_counts()) == live, k
    g.close()
