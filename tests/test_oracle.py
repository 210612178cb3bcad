"""CPU checks of the oracle: against the reference's own C code (oracle/_ref)
and against exact identities of the restated algorithms."""
import ctypes

import numpy as np
import pytest

from ctca_b200 import inputs
from ctca_b200.emses import PARTICLE_DTYPE
from oracle import oracle as O


def small_case(n=(8, 8, 8), ppc=(4, 4), seed=7, e=True, b0=(0.0, 0.0, 0.2)):
    c = inputs.workload_case(1)
    c.n = n
    c.species[0].ppc, c.species[1].ppc = ppc
    c.kmax = 2 * np.pi / min(n) * 2
    c.seed = seed
    c.b0 = b0
    if not e:
        c.e_modes = 0
        c.e0 = (0.0, 0.0, 0.0)
    return c


# ---- the reference's C sources, compiled in oracle/_ref ------------------
def ref_or_skip():
    L = O.ref_lib()
    if L is None:
        pytest.skip("oracle/_ref not built (reference sources absent)")
    return L


def test_ref_mt19937_known_answer():
    # MT19937 reference output: init_genrand(5489) -> first genrand_int32 3499211612
    L = ref_or_skip()
    L.mtrand_int32_.restype = ctypes.c_int
    s = ctypes.c_int(5489)
    L.mt_init_(ctypes.byref(s))
    assert L.mtrand_int32_() & 0xFFFFFFFF == 3499211612


def test_ranu0_stream_is_53bit_uniform():
    ref_or_skip()
    u = O.ranu0_stream(10, 2000)  # seed (myid+1)*10 of inital.F90:707-708
    assert (u >= 0).all() and (u < 1).all()
    assert abs(u.mean() - 0.5) < 0.03
    assert np.all(np.floor(u * 2.0 ** 53) == u * 2.0 ** 53)


def test_canonical_order_is_sorted_under_the_reference_comparator():
    """After our stable cell-key sort, every consecutive pair satisfies the
    reference comparator (int)(a->z - b->z) <= 0 (psort-struct.c:15-20), and
    the reference's own particle_sort_ leaves z cells non-decreasing."""
    L = ref_or_skip()
    case = small_case()
    cfg = inputs.make_config(case)
    p, tp = inputs.make_particles(case)
    o = O.Oracle(cfg, p, tp, inputs.make_fields(case))
    o.spsort()
    seg = o.pbuf[: tp[0]]
    dz = seg["z"][:-1] - seg["z"][1:]
    assert np.all(np.trunc(dz) <= 0)
    ref = p[: tp[0]].copy()
    n = ctypes.c_int(int(tp[0]))
    L.particle_sort_(ref.ctypes.data, ctypes.byref(n))
    assert sorted(ref["z"].tolist()) == sorted(p[: tp[0]]["z"].tolist())  # a permutation
    assert np.all(np.trunc(ref["z"][:-1] - ref["z"][1:]) <= 0)


# ---- exact identities ------------------------------------------------------
def test_cic_charge_sum_is_exact():
    case = small_case()
    cfg = inputs.make_config(case)
    p, tp = inputs.make_particles(case)
    o = O.Oracle(cfg, p, tp, inputs.make_fields(case))
    o.charge(0)
    total = tp[0] * cfg.q[0] + tp[1] * cfg.q[1]
    assert abs(o.f["rho"].sum() - total) < 1e-12
    o.reduce_rho()
    interior = o.f["rho"][1:-2, 1:-2, 1:-2, 0]  # nodes 0..n-1 carry every image once
    assert abs(interior.sum() - total) < 1e-12


def test_boris_rotation_keeps_speed_without_e():
    case = small_case(e=False, b0=(0.3, -0.2, 0.5))
    cfg = inputs.make_config(case)
    p, tp = inputs.make_particles(case)
    o = O.Oracle(cfg, p, tp, inputs.make_fields(case))
    o.grdcrt()
    v0 = np.sqrt(p["vx"] ** 2 + p["vy"] ** 2 + p["vz"] ** 2)
    o.psolve2(2)
    v1 = np.sqrt(o.pbuf["vx"] ** 2 + o.pbuf["vy"] ** 2 + o.pbuf["vz"] ** 2)
    assert np.max(np.abs(v1 - v0) / v0) < 1e-14


def cic_nodes(x):
    i = np.floor(x).astype(int)
    f = x - i
    out = {}
    for di in (0, 1):
        for dj in (0, 1):
            for dk in (0, 1):
                w = (f[0] if di else 1 - f[0]) * (f[1] if dj else 1 - f[1]) * (f[2] if dk else 1 - f[2])
                out[(i[0] + di, i[1] + dj, i[2] + dk)] = w
    return out


@pytest.mark.parametrize("seed", range(6))
def test_zigzag_residual_is_the_cubic_term(seed):
    """For one particle, rho(n+1) - rho(n) + 2 div J equals, node by node, the
    cubic term of the trilinear product difference, q*da*db*dc/4 times the
    corner signs, summed over the (one or two) zigzag segments.  This pins
    every index and weight of the 24 scatter-adds of psolve1.F90:759-789."""
    rng = np.random.default_rng(seed)
    case = small_case(e=False, b0=(0.0, 0.0, 0.0))
    case.species = [case.species[0]]
    cfg = inputs.make_config(case)
    p = np.zeros(1, dtype=PARTICLE_DTYPE)
    x0 = rng.uniform(2.0, 5.0, 3)
    v = rng.uniform(-0.45, 0.45, 3)
    p["x"], p["y"], p["z"] = x0
    p["vx"], p["vy"], p["vz"] = v
    o = O.Oracle(cfg, p, [1], inputs.make_fields(case))
    o.grdcrt()
    o.charge(0)
    r0 = o.f["rho"].copy()
    o.psolve1(2, 0)
    o.charge(0)
    r1 = o.f["rho"]
    a = o.f["aj"]
    x1 = np.array([o.pbuf["x"][0], o.pbuf["y"][0], o.pbuf["z"][0]])
    # zigzag relay point
    ib, ia = np.floor(x0), np.floor(x1)
    xr = np.where(ib == ia, 0.5 * (x0 + x1), np.maximum(ib, ia))
    expect = {}
    for s0, s1 in ((x0, xr), (xr, x1)):
        base = np.floor(np.minimum(s0, s1) + 0 * s0)
        cell = np.floor(0.5 * (s0 + s1))
        f0, f1 = s0 - cell, s1 - cell
        d = f1 - f0
        for di in (0, 1):
            for dj in (0, 1):
                for dk in (0, 1):
                    sign = (1 if di else -1) * (1 if dj else -1) * (1 if dk else -1)
                    key = (int(cell[0]) + di, int(cell[1]) + dj, int(cell[2]) + dk)
                    expect[key] = expect.get(key, 0.0) + sign * cfg.q[0] * d[0] * d[1] * d[2] / 4.0
    for k in range(1, 7):
        for j in range(1, 7):
            for i in range(1, 7):
                div = (a[k + 4, j + 4, i + 4, 0] - a[k + 4, j + 4, i + 3, 0] + a[k + 4, j + 4, i + 4, 1]
                       - a[k + 4, j + 3, i + 4, 1] + a[k + 4, j + 4, i + 4, 2] - a[k + 3, j + 4, i + 4, 2])
                res = r1[k + 1, j + 1, i + 1, 0] - r0[k + 1, j + 1, i + 1, 0] + 2.0 * div
                assert abs(res - expect.get((i, j, k), 0.0)) < 1e-15, (i, j, k)


def test_reduce_rho_sums_periodic_images():
    case = small_case()
    cfg = inputs.make_config(case)
    rng = np.random.default_rng(3)
    raw = np.zeros((11, 11, 11, 1))
    raw[1:10, 1:10, 1:10, 0] = rng.normal(size=(9, 9, 9))  # nodes 0..n deposited
    o = O.Oracle(cfg, np.zeros(0, dtype=PARTICLE_DTYPE), [0, 0], inputs.make_fields(case))
    o.f["rho"][...] = raw
    o.reduce_rho()
    folded = np.zeros((8, 8, 8))
    for k in range(9):
        for j in range(9):
            for i in range(9):
                folded[k % 8, j % 8, i % 8] += raw[k + 1, j + 1, i + 1, 0]
    got = o.f["rho"][1:9, 1:9, 1:9, 0]
    assert np.allclose(got, folded, rtol=0, atol=1e-12)
    # node n repeats node 0
    assert np.allclose(o.f["rho"][9, 1:10, 1:10, 0], o.f["rho"][1, 1:10, 1:10, 0], atol=1e-12)


def test_spsort_is_stable_and_keyed():
    case = small_case()
    case.sort_tile = (4, 4, 2)
    cfg = inputs.make_config(case)
    p, tp = inputs.make_particles(case)
    rng = np.random.default_rng(5)
    perm = np.concatenate([rng.permutation(tp[0]), tp[0] + rng.permutation(tp[1])])
    p = p[perm]
    p["pid"] = np.arange(p.size) % 1000
    o = O.Oracle(cfg, p, tp, inputs.make_fields(case))
    keys_before = o.sort_keys()
    o.spsort()
    keys = o.sort_keys()
    for s, (a, b) in enumerate(((0, tp[0]), (tp[0], tp[0] + tp[1]))):
        assert np.all(np.diff(keys[a:b]) >= 0)
        order = np.argsort(keys_before[a:b], kind="stable")
        assert np.array_equal(o.pbuf[a:b], p[a:b][order])


def test_compact_keeps_order():
    case = small_case()
    cfg = inputs.make_config(case)
    p, tp = inputs.make_particles(case)
    p["nid"][::3] = -1
    o = O.Oracle(cfg, p, tp, inputs.make_fields(case))
    o.compact()
    keep0 = p[: tp[0]][p[: tp[0]]["nid"] != -1]
    keep1 = p[tp[0]:][p[tp[0]:]["nid"] != -1]
    assert np.array_equal(o.pbuf, np.concatenate([keep0, keep1]))
    assert list(o.totalp) == [keep0.size, keep1.size]


def test_hash_uniforms():
    u = np.array([O.hash_u01(1, 2, i) for i in range(4000)])
    assert (u >= 0).all() and (u < 1).all() and abs(u.mean() - 0.5) < 0.02


def test_background_charge_from_surface_counts():
    """orc_background: one count on a face cell puts q/4 on each of the
    four nodes of that face cell; any counts give total charge sum(q * count);
    rho(0:n) gets rhobk added, or replaced with replace."""
    case = small_case(n=(12, 10, 14))
    box = dict(geotype=0, ncond=1, xlpc=3.0, xupc=7.0, ylpc=2.0, yupc=5.0, zlpc=4.0, zupc=9.0, sqdscaled=1.0)
    case.bodies = [box]
    cfg = inputs.make_config(case)
    p, tp = inputs.make_particles(case)
    o = O.Oracle(cfg, p[:0], [0, 0], inputs.make_fields(case))
    off = np.zeros(6 * 4, dtype=np.int64)
    nsurf = int(O.lib().orc_surface_layout(ctypes.byref(cfg), off.ctypes.data))
    assert nsurf == 2 * (3 * 5 + 4 * 5 + 4 * 3)
    lo, hi = (3, 2, 4), (7, 5, 9)
    # +y face (f = 3), cell (u, v) = (1, 2): x in [4, 5], z in [6, 7], y = 5
    surf = np.zeros((cfg.nspec, nsurf), dtype=np.int64)
    surf[0, off[3] + 1 + 4 * 2] = 1
    o.background(surf=surf)
    rb = o.f["rhobk"][..., 0]
    nz_idx = np.argwhere(rb != 0)
    got = {(int(k) - 1, int(j) - 1, int(i) - 1) for k, j, i in nz_idx}
    assert got == {(6, 5, 4), (6, 5, 5), (7, 5, 4), (7, 5, 5)}  # (k, j, i)
    assert np.all(rb[rb != 0] == cfg.q[0] * 0.25)
    # random counts: the total charge, and rho += rhobk on the nodes 0..n
    rng = np.random.default_rng(3)
    surf = rng.integers(-3, 9, size=(cfg.nspec, nsurf))
    o.f["rho"][...] = rng.random(o.f["rho"].shape)
    rho0 = o.f["rho"].copy()
    o.background(surf=surf)
    want = sum(cfg.q[s] * surf[s].sum() for s in range(cfg.nspec))
    assert abs(o.f["rhobk"].sum() - want) <= 1e-12 * np.abs(cfg.q[:2]).sum() * np.abs(surf).sum()
    inner = (slice(1, cfg.nz + 2), slice(1, cfg.ny + 2), slice(1, cfg.nx + 2))
    assert np.array_equal(o.f["rho"][inner], rho0[inner] + o.f["rhobk"][inner])
    o.background(surf=surf, replace=True)
    assert np.array_equal(o.f["rho"][inner], o.f["rhobk"][inner])


def test_zigzag_one_sums_to_psolve1():
    """orc_zigzag_one (the checker's per-particle zigzag) summed over every
    particle equals psolve1's folded current on the nodes 0..n-1 of a
    periodic grid with no fields (so a = b + v ustep), many particles
    crossing faces."""
    case = small_case(n=(8, 6, 5), e=False, b0=(0.0, 0.0, 0.0))
    case.species[0].vth *= 8
    cfg = inputs.make_config(case)
    p, tp = inputs.make_particles(case)
    o = O.Oracle(cfg, p, tp, inputs.make_fields(case) * 0.0)
    o.grdcrt()
    o.f["aj"][...] = 0.0
    o.psolve1(2, 0)
    o.reduce_aj()
    J = np.zeros((cfg.nx * cfg.ny * cfg.nz, 3))
    L = O.lib()
    for m in range(p.size):
        b = np.array([p[f][m] for f in "xyz"])
        a = b + 2.0 * np.array([p[f][m] for f in ("vx", "vy", "vz")])
        L.orc_zigzag_one(ctypes.byref(cfg), 2, cfg.q[int(p["spec"][m]) - 1], b.ctypes.data, a.ctypes.data,
                         J.ctypes.data)
    got = J.reshape(cfg.nz, cfg.ny, cfg.nx, 3)
    want = o.f["aj"][4:4 + cfg.nz, 4:4 + cfg.ny, 4:4 + cfg.nx]
    crossing = np.any(np.floor(np.stack([p[f] for f in "xyz"], 1)) != np.floor(np.stack(
        [p[f] + 2 * p[v] for f, v in zip("xyz", ("vx", "vy", "vz"))], 1)), 1)
    assert crossing.sum() > 50
    assert np.linalg.norm(got - want) <= 1e-12 * np.linalg.norm(want)
