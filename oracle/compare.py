"""TEST INFRASTRUCTURE ONLY: per-quantity errors of the FP32 / fixed-point
form against the FP64 oracle.

Used by tests/ and by bench.py's accuracy report, always as the checker.
The FP32 form and the oracle start a step from the same state (the FP32
form's own particles as FP64 records, emsesg_fx_store), so a difference in
a particle's cell after the step can only come from FP32 rounding of a
position that ends next to a cell face.  Such particles are counted, and a
cell difference of any particle farther than `band` from every face counts
as a failure of exactness.

The sort permutation is the definition of the FP32 tile sort: live particles
ordered by the tile-major cell key, equal cells in the order (source tile,
warp, row, lane) of the thread-major layout of the previous sort (the sorted
rank q of a tile of n particles sits in row q % L, column q / L,
L = ceil(n / row slots); a warp is 32 consecutive columns).
"""
from __future__ import annotations

import numpy as np

FP32_ULP = 2.0 ** -23   # one FP32 ulp of an in-cell offset in [0.5, 1)
BAND = 4 * FP32_ULP     # "next to a face": within four ulps


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def max_rel(a, b) -> float:
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    mb = np.max(np.abs(b)) if b.size else 0.0
    return float(np.max(np.abs(a - b)) / (mb if mb > 0 else 1.0)) if b.size else 0.0


def _cells(cfg, p):
    return np.stack([np.floor(p[f]).astype(np.int64) for f in "xyz"], 1)


def particle_errors(cfg, pg, po, band: float = BAND) -> dict:
    """Errors of the FP32 form's records pg against the oracle's po (same
    particles, same order, after the same step from the same state)."""
    ext = np.array([cfg.nx, cfg.ny, cfg.nz], dtype=np.float64)
    alive_g, alive_o = pg["nid"] != -1, po["nid"] != -1
    m = alive_g & alive_o
    a, b = pg[m], po[m]
    out = {"particles": int(po.size), "alive": int(alive_o.sum()),
           "alive_mismatch": int((alive_g != alive_o).sum())}
    dpos = np.stack([a[f] - b[f] for f in "xyz"], 1)
    dpos = dpos - ext * np.round(dpos / ext)  # a periodic wrap is no error
    out["pos_max_abs"] = float(np.max(np.abs(dpos))) if dpos.size else 0.0
    out["pos_rms"] = float(np.sqrt(np.mean(np.sum(dpos ** 2, 1)))) if dpos.size else 0.0
    vg = np.stack([a[f] for f in ("vx", "vy", "vz")], 1)
    vo = np.stack([b[f] for f in ("vx", "vy", "vz")], 1)
    out["vel_max_rel"] = max_rel(vg, vo)
    out["vel_l2_rel"] = rel_l2(vg, vo)
    cg = _cells(cfg, a) % ext.astype(np.int64)
    co = _cells(cfg, b) % ext.astype(np.int64)
    mis = np.any(cg != co, 1)
    frac = np.stack([b[f] - np.floor(b[f]) for f in "xyz"], 1)
    near = np.any((frac < band) | (frac > 1.0 - band), 1)
    out["cell_mismatch"] = int(mis.sum())
    out["cell_mismatch_off_band"] = int((mis & ~near).sum())
    out["near_face"] = int(near.sum())
    out["band"] = band
    out["mismatched"] = np.flatnonzero(m)[mis]  # indices into the records
    return out


def nodes(cfg, a):
    """The nodes 0..n of every axis of a rho-layout (guard 1) or aj-layout
    (guard 4) array, numpy shape (z, y, x[, c]): the field the reference's
    solver and rhoupd use.  The guard layers are left out: after a periodic
    fold they keep partial sums that depend on which side of a periodic face
    a particle is stored, and a particle that ends within an FP32 ulp of that
    face is stored on one side by the FP32 form and on the other by FP64."""
    nx, ny, nz = cfg.nx, cfg.ny, cfg.nz
    lo = (a.shape[0] - nz - 1) // 2  # 1 for rho, 4 for aj
    return a[lo:lo + nz + 1, lo:lo + ny + 1, lo:lo + nx + 1]


def field_errors(g, o, cfg=None) -> dict:
    """Relative L2 and max errors of a field, on the nodes 0..n when cfg is
    given (see nodes), else over the whole array."""
    if cfg is not None:
        g, o = nodes(cfg, g), nodes(cfg, o)
    return {"l2_rel": rel_l2(g, o), "max_rel": max_rel(g, o)}


def tile_key(cfg, tile, p):
    """Tile-major cell key and tile index of records p (tile: cells a side)."""
    i, j, k = (np.floor(p[f]).astype(np.int64) % n for f, n in zip("xyz", (cfg.nx, cfg.ny, cfg.nz)))
    nt = [-(-n // t) for n, t in zip((cfg.nx, cfg.ny, cfg.nz), tile)]
    tid = i // tile[0] + nt[0] * (j // tile[1] + nt[1] * (k // tile[2]))
    lin = i % tile[0] + tile[0] * (j % tile[1] + tile[1] * (k % tile[2]))
    return tid * (tile[0] * tile[1] * tile[2]) + lin, tid


def sort_order(cfg, tile, row_slots, before, after, keys=None):
    """The permutation of one species' tile sort: `before` are its records
    in the order of the previous sort (cells of that sort), `after` the same
    particles moved by the steps since; returns the indices of the live
    particles of `after` in sorted order.  `keys` overrides the cell keys of
    `after` (e.g. the oracle's)."""
    _, t0 = tile_key(cfg, tile, before)
    ntile = int(t0.max()) + 1 if t0.size else 0
    counts = np.bincount(t0, minlength=ntile)
    starts = np.concatenate([[0], np.cumsum(counts)])
    q = np.arange(before.size) - starts[t0]
    L = -(-counts[t0] // row_slots)
    col, row = q // L, q % L
    src = np.lexsort((col % 32, row, col // 32, t0))  # (tile, warp, row, lane)
    order_pos = np.empty(before.size, dtype=np.int64)
    order_pos[src] = np.arange(before.size)
    live = after["nid"] != -1
    key1 = tile_key(cfg, tile, after)[0] if keys is None else keys
    idx = np.flatnonzero(live)
    return idx[np.lexsort((order_pos[idx], key1[idx]))]


def cell_histogram(cfg, p) -> np.ndarray:
    c = _cells(cfg, p[p["nid"] != -1]) % np.array([cfg.nx, cfg.ny, cfg.nz])
    lin = c[:, 0] + cfg.nx * (c[:, 1] + cfg.ny * c[:, 2])
    return np.bincount(lin, minlength=cfg.nx * cfg.ny * cfg.nz)


def continuity_residual(cfg, rho_old, rho_new, aj) -> float:
    """max over the nodes 0..n of |rho_new - rho_old + 2 div J| (rhoupd.F90:
    41-49), FP64; rho arrays of the rho layout (guard 1), aj of the aj layout
    (guard 4), numpy shape (z, y, x[, c])."""
    nx, ny, nz = cfg.nx, cfg.ny, cfg.nz
    r0 = rho_old.reshape(nz + 3, ny + 3, nx + 3)[1:nz + 2, 1:ny + 2, 1:nx + 2]
    r1 = rho_new.reshape(nz + 3, ny + 3, nx + 3)[1:nz + 2, 1:ny + 2, 1:nx + 2]
    j = aj.reshape(nz + 9, ny + 9, nx + 9, 3)
    jx = j[4:nz + 5, 4:ny + 5, 4:nx + 5, 0] - j[4:nz + 5, 4:ny + 5, 3:nx + 4, 0]
    jy = j[4:nz + 5, 4:ny + 5, 4:nx + 5, 1] - j[4:nz + 5, 3:ny + 4, 4:nx + 5, 1]
    jz = j[4:nz + 5, 4:ny + 5, 4:nx + 5, 2] - j[3:nz + 4, 4:ny + 5, 4:nx + 5, 2]
    return float(np.max(np.abs(r1 - (r0 - ((jx + jy) + jz) * 2.0))))


def zigzag_correction(cfg, start, g_end, o_end, idx, ustep: int = 2) -> np.ndarray:
    """The current that particles `idx` deposit with the FP32 form's end
    point (g_end) minus the current with the oracle's (o_end), from the same
    start (FP64 zigzag of oracle/adjoint.cpp, periodic grid): numpy
    (nz, ny, nx, 3) on the nodes 0..n-1.  Added to the oracle's J it gives
    the oracle's J for the cells the FP32 form took."""
    import ctypes
    from . import oracle as O
    L = O.lib()
    J = np.zeros((cfg.nx * cfg.ny * cfg.nz, 3))
    ext = np.array([cfg.nx, cfg.ny, cfg.nz], dtype=np.float64)
    for m in np.asarray(idx, dtype=np.int64):
        b = np.array([start[f][m] for f in "xyz"])
        q = cfg.q[int(start["spec"][m]) - 1]
        for end, sign in ((g_end, 1.0), (o_end, -1.0)):
            d = np.array([end[f][m] for f in "xyz"]) - b
            a = b + (d - ext * np.round(d / ext))
            L.orc_zigzag_one(ctypes.byref(cfg), ustep, sign * q, b.ctypes.data, a.ctypes.data, J.ctypes.data)
    return J.reshape(cfg.nz, cfg.ny, cfg.nx, 3)


def j_error_corrected(cfg, jg, jo, start, g_end, o_end, idx) -> tuple[float, float]:
    """Relative L2 error of the FP32 form's J (aj layout) against the
    oracle's on the nodes 0..n-1 of a periodic grid: as is, and with the
    oracle's J moved to the cells the FP32 form took for the particles
    `idx` (zigzag_correction)."""
    nx, ny, nz = cfg.nx, cfg.ny, cfg.nz
    g = jg.reshape(nz + 9, ny + 9, nx + 9, 3)[4:4 + nz, 4:4 + ny, 4:4 + nx]
    o = jo.reshape(nz + 9, ny + 9, nx + 9, 3)[4:4 + nz, 4:4 + ny, 4:4 + nx]
    corr = zigzag_correction(cfg, start, g_end, o_end, idx) if len(idx) else 0.0
    return rel_l2(g, o), rel_l2(g, o + corr)


def near_faces(cfg, start, end, bodies=(), band: float = BAND, tie: float = 1e-5) -> np.ndarray:
    """Particles whose FP64 move start -> end comes within `band` of a
    decision that FP32 rounding can flip: an end point within `band` of an
    integer plane on any axis (cell faces, the faces of box bodies with
    integer bounds, the outer faces), or, for an end point inside a box (the
    absorption test, inclusive bounds), two face entry times within `tie` of
    each other (the face crossed last picks the surface cell).  bodies:
    (lo[3], hi[3]) integer boxes."""
    e = np.stack([end[f] for f in "xyz"], 1)
    s = np.stack([start[f] for f in "xyz"], 1)
    # (records of dead particles may hold no number: they compare false)
    with np.errstate(divide="ignore", invalid="ignore"):
        frac = e - np.floor(e)
        near = np.any((frac < band) | (frac > 1.0 - band), 1)
        for lo, hi in bodies:
            lo, hi = np.asarray(lo, float), np.asarray(hi, float)
            inside = np.all((e >= lo) & (e <= hi), 1)
            t = np.where(s < lo, (lo - s) / (e - s), np.where(s > hi, (hi - s) / (e - s), -1.0))
            ts = np.sort(t, 1)
            close = (ts[:, 1] >= 0) & (ts[:, 2] - ts[:, 1] < tie)
            near |= inside & close
    return near


def near_curved(end, bodies, band: float = 1e-5) -> np.ndarray:
    """Particles whose FP64 end point lies within `band` (cells) of the
    surface of a cylinder or a sphere, where FP32 rounding of the position
    or of the squared distance can flip the absorption test of
    psolve1.F90:684-712.  bodies: emsesg_body-like dicts (geotype 2 with
    cyl_align, cyl_axis, cyl_edge, radius; geotype 3 with sph_center,
    radius); other geotypes are skipped."""
    e = np.stack([end[f] for f in "xyz"], 1)
    near = np.zeros(e.shape[0], dtype=bool)
    for b in bodies:
        if b["geotype"] not in (2, 3):
            continue
        r = float(b["radius"])
        if b["geotype"] == 3:
            d = np.sqrt(((e - np.asarray(b["sph_center"], float)) ** 2).sum(1))
            near |= np.abs(d - r) < band
        elif b["geotype"] == 2:
            a0 = int(b["cyl_align"]) - 1
            a1, a2 = (a0 + 1) % 3, (a0 + 2) % 3
            d = np.hypot(e[:, a1] - b["cyl_axis"][0], e[:, a2] - b["cyl_axis"][1])
            lo, hi = b["cyl_edge"]
            ax = e[:, a0]
            within = (ax >= lo - band) & (ax <= hi + band)
            near |= within & (np.abs(d - r) < band)
            near |= (d < r + band) & ((np.abs(ax - lo) < band) | (np.abs(ax - hi) < band))
    return near
