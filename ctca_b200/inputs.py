"""Seeded synthetic inputs in the reference's internal units.

The benchmark configurations of the EMSES particle path are stated in
normalized units (c = 1, omega_pe = 1, dx = 1, dt = 0.5).  The reference
converts them to internal units in rescal (src/main/rescal.F90:44-81 and
:126-169): with dth = dt/2 and qm1 = qm(1) (electrons, -1)

    position  x r      renr = 1/dr
    velocity  x renv   renv = dth/dr
    E         x rene   rene = qm1*dth**2/dr
    B         x renb   renb = qm1*dth
    q         x renq   renq = qm1*(dth/dr)**2/dr
    qm        / qm1
    mass      x renm   renm = (qm1*dth/dr)**2/dr

and sets the macro-particle charge from the plasma frequency,
q(is) = wp(is)**2 * V / npin(is) / qm(is) (src/main/inital.F90:231), with
rm(is) = q(is)/qm(is) (:271).  Ions get the charge that neutralises the
electrons.

Fields are staggered on the Yee grid as the reference stores eb
(grdcrt.F90:156-230): EX at (i+1/2, j, k), BX at (i, j+1/2, k+1/2), and so on.
Fluctuations are sums of seeded Fourier modes A*u*cos(k.r + phi) with integer
wave numbers, so they are periodic on the grid; guards are periodic copies, as
oh3_exchange_borders leaves them.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .emses import ISPEC, PARTICLE_DTYPE, Config, Plasma, field_extents


@dataclass
class Species:
    ppc: int
    qm: float            # normalized charge-to-mass ratio (electrons -1)
    vth: float           # normalized thermal speed
    drift: tuple = (0.0, 0.0, 0.0)
    npbnd: tuple = (0, 0, 0)


@dataclass
class Case:
    n: tuple
    species: list
    dt: float = 0.5
    b0: tuple = (0.0, 0.0, 0.0)
    e0: tuple = (0.0, 0.0, 0.0)
    e_modes: int = 0
    e_amp: float = 0.0
    b_modes: int = 0
    b_amp: float = 0.0
    kmax: float = 0.0     # |k| cap of the modes (radians per cell)
    nfbnd: tuple = (0, 0, 0)
    seed: int = 1001
    sort_tile: tuple = (0, 0, 0)
    capacity_factor: float = 1.0
    bodies: list = field(default_factory=list)


def units(dt: float = 0.5, dr: float = 1.0, qm1: float = -1.0) -> dict:
    dth = dt / 2.0
    return {
        "dth": dth,
        "renv": dth / dr,
        "rene": qm1 * dth * dth / dr,
        "renb": qm1 * dth,
        "renq": qm1 * (dth / dr) ** 2 / dr,
        "renm": (qm1 * dth / dr) ** 2 / dr,
        "renrho": qm1 * dth * dth,
        "renj": qm1 * dth ** 3 / dr,
        "qm1": qm1,
    }


def workload_case(idx: int, scale: float = 1.0) -> Case:
    """The benchmark workloads (normalized units):
    1: 32^3 periodic, 2 species x 16 ppc, mass ratio 100, B0 along z, E0 plus
       4 Fourier modes (the CPU-sized case);
    2: 128^3 periodic, 2 species x 64 ppc, mass ratio 1836, ion drift, 8 E
       and 8 B modes (the headline particle step);
    3: 256x256x512, open z, 2 species x 24 ppc drifting along -z past a
       32x32x16 conducting box (the body workload);
    4: 64^3 periodic, the plasma of case 1 at 32 ppc (the adjoint workload).
    `scale` shrinks the grid of cases 2-4."""
    if idx == 1:
        return Case(n=(32, 32, 32),
                    species=[Species(16, -1.0, 0.05), Species(16, 1.0 / 100.0, 0.005)],
                    b0=(0.0, 0.0, 0.2), e0=(1e-3, 0.0, 0.0), e_modes=4, e_amp=1e-3,
                    kmax=4 * 2 * math.pi / 32, seed=1001)
    if idx == 2:
        n = max(8, int(round(128 * scale)))
        ppc = 64
        return Case(n=(n, n, n),
                    species=[Species(ppc, -1.0, 0.05),
                             Species(ppc, 1.0 / 1836.0, 0.05 / math.sqrt(1836.0), drift=(0.01, 0.0, 0.0))],
                    b0=(0.0, 0.0, 0.1), e_modes=8, e_amp=1e-3, b_modes=8, b_amp=1e-3,
                    kmax=4 * 2 * math.pi / n, seed=1002, sort_tile=(8, 8, 8))
    if idx == 3:
        # the body workload: solar wind along -z past a conducting box
        nx, ny, nz = (max(16, int(round(256 * scale))), max(16, int(round(256 * scale))),
                      max(32, int(round(512 * scale))))
        c = Case(n=(nx, ny, nz),
                 species=[Species(24, -1.0, 0.05, drift=(0.0, 0.0, -0.08), npbnd=(0, 0, 2)),
                          Species(24, 1.0 / 100.0, 0.005, drift=(0.0, 0.0, -0.08), npbnd=(0, 0, 2))],
                 b0=(0.05, 0.0, 0.1), nfbnd=(0, 0, 1), seed=1003, sort_tile=(8, 8, 8))
        bx, by, bz = max(2, int(round(32 * scale))), max(2, int(round(32 * scale))), max(2, int(round(16 * scale)))
        x0, y0, z0 = (nx - bx) // 2, (ny - by) // 2, (nz - bz) // 2
        c.bodies = [dict(geotype=0, ncond=1, xlpc=float(x0), xupc=float(x0 + bx), ylpc=float(y0),
                         yupc=float(y0 + by), zlpc=float(z0), zupc=float(z0 + bz), sqdscaled=1.0)]
        return c
    if idx == 4:
        # the adjoint workload: 64^3, the plasma of case 1 at 32 ppc
        c = workload_case(1)
        n = max(8, int(round(64 * scale)))
        c.n = (n, n, n)
        for sp in c.species:
            sp.ppc = 32
        c.kmax = 4 * 2 * math.pi / n
        c.seed = 1004
        c.sort_tile = (8, 8, 8)
        return c
    raise ValueError(f"no workload case {idx}")


def charges(case: Case) -> tuple[list, list, list]:
    """Normalized q, qm, rm per species (inital.F90:231, :271)."""
    q, qm, rm = [], [], []
    e = case.species[0]
    qe = 1.0 * 1.0 / e.ppc / e.qm  # wp=1, V/npin = 1/ppc
    for s in case.species:
        if s is e:
            qs = qe
        elif s.ppc > 0:
            qs = -qe * e.ppc / s.ppc  # neutralising
        else:
            qs = -qe  # a species without particles: any finite charge
        q.append(qs)
        qm.append(s.qm)
        rm.append(qs / s.qm)
    return q, qm, rm


def make_config(case: Case, capacity: list | None = None) -> Config:
    u = units(case.dt, 1.0, case.species[0].qm)
    c = Config()
    c.nx, c.ny, c.nz = case.n
    c.nspec = len(case.species)
    for d in range(3):
        c.nfbnd[d] = case.nfbnd[d]
        c.sort_tile[d] = case.sort_tile[d]
    q, qm, rm = charges(case)
    ncell = case.n[0] * case.n[1] * case.n[2]
    for i, s in enumerate(case.species):
        for d in range(3):
            c.npbnd[i][d] = s.npbnd[d]
        c.q[i] = q[i] * u["renq"]
        c.qm[i] = qm[i] / u["qm1"]
        c.rm[i] = rm[i] * u["renm"]
        cap = capacity[i] if capacity is not None else int(math.ceil(ncell * s.ppc * case.capacity_factor))
        c.capacity[i] = cap
    for d in range(3):
        c.e0[d] = case.e0[d] * u["rene"]
        c.b0[d] = case.b0[d] * u["renb"]
    c.npc = len(case.bodies)
    c.line_mode = 0
    for i, b in enumerate(case.bodies):
        for k, v in b.items():
            if isinstance(v, (list, tuple)):
                arr = getattr(c.body[i], k)
                for j, x in enumerate(v):
                    arr[j] = x
            else:
                setattr(c.body[i], k, v)
    c.rng_mode = 0
    c.rng_seed = case.seed
    return c


def _modes(rng: np.random.Generator, n: tuple, count: int, kmax: float, transverse: bool):
    out = []
    mmax = [int(math.floor(kmax * n[d] / (2 * math.pi))) for d in range(3)]
    while len(out) < count:
        m = np.array([rng.integers(-mmax[d], mmax[d] + 1) for d in range(3)], dtype=float)
        if not m.any():
            continue
        k = 2 * math.pi * m / np.array(n, dtype=float)
        if np.linalg.norm(k) > kmax * (1 + 1e-12):
            continue
        pol = rng.normal(size=3)
        if transverse:
            pol -= pol.dot(k) / k.dot(k) * k
        pol /= np.linalg.norm(pol)
        out.append((k, pol, rng.uniform(0, 2 * math.pi)))
    return out


def make_fields(case: Case) -> np.ndarray:
    """eb(6, -1:nx+1, -1:ny+1, -1:nz+1) in internal units, numpy shape
    (nz+3, ny+3, nx+3, 6); periodic guards."""
    u = units(case.dt, 1.0, case.species[0].qm)
    nx, ny, nz = case.n
    rng = np.random.default_rng(case.seed)
    emodes = _modes(rng, case.n, case.e_modes, case.kmax, False) if case.e_modes else []
    bmodes = _modes(rng, case.n, case.b_modes, case.kmax, True) if case.b_modes else []
    # interior grid indices 0..n-1; positions of each staggered component
    i = np.arange(nx, dtype=float)[None, None, :]
    j = np.arange(ny, dtype=float)[None, :, None]
    k = np.arange(nz, dtype=float)[:, None, None]
    h = 0.5
    offs = {0: (h, 0, 0), 1: (0, h, 0), 2: (0, 0, h), 3: (0, h, h), 4: (h, 0, h), 5: (h, h, 0)}
    inner = np.zeros((nz, ny, nx, 6))
    for comp in range(6):
        ox, oy, oz = offs[comp]
        modes, amp, ren = (emodes, case.e_amp, u["rene"]) if comp < 3 else (bmodes, case.b_amp, u["renb"])
        acc = np.zeros((nz, ny, nx))
        for kv, pol, ph in modes:
            arg = kv[0] * (i + ox) + kv[1] * (j + oy) + kv[2] * (k + oz) + ph
            acc = acc + amp * pol[comp % 3] * np.cos(arg)
        inner[..., comp] = acc * ren
    # periodic guard fill (-1 .. n+1)
    ix = np.arange(-1, nx + 2) % nx
    iy = np.arange(-1, ny + 2) % ny
    iz = np.arange(-1, nz + 2) % nz
    eb = inner[np.ix_(iz, iy, ix)]
    return np.ascontiguousarray(eb)


def make_particles(case: Case, ppc_override: list | None = None, cells: int | None = None):
    """ppc particles per cell per species at cell + U[0,1)^3 (x fastest cell
    order), Maxwellian velocities plus drift, internal units.  `cells` keeps
    only the first `cells` cells (a bounded sample of the same plasma)."""
    u = units(case.dt, 1.0, case.species[0].qm)
    nx, ny, nz = case.n
    ncell = nx * ny * nz if cells is None else min(cells, nx * ny * nz)
    rng = np.random.default_rng(case.seed + 17)
    parts, totalp = [], []
    for isp, s in enumerate(case.species):
        ppc = s.ppc if ppc_override is None else ppc_override[isp]
        n = ncell * ppc
        cell = np.repeat(np.arange(ncell, dtype=np.int64), ppc)
        p = np.zeros(n, dtype=PARTICLE_DTYPE)
        p["x"] = (cell % nx) + rng.random(n)
        p["y"] = ((cell // nx) % ny) + rng.random(n)
        p["z"] = (cell // (nx * ny)) + rng.random(n)
        for d, name in enumerate(("vx", "vy", "vz")):
            p[name] = (rng.normal(0.0, s.vth, n) + s.drift[d]) * u["renv"]
        p["spec"] = isp + 1
        parts.append(p)
        totalp.append(n)
    return np.concatenate(parts), np.array(totalp, dtype=np.int64)


def plasma(case: Case, seed: int | None = None) -> Plasma:
    """Device-loader parameters (emsesg_load_plasma) of the same plasma."""
    u = units(case.dt, 1.0, case.species[0].qm)
    pl = Plasma()
    for i, s in enumerate(case.species):
        pl.ppc[i] = s.ppc
        pl.vth[i] = s.vth * u["renv"]
        for d in range(3):
            pl.vdrift[i][d] = s.drift[d] * u["renv"]
    pl.seed = case.seed if seed is None else seed
    return pl


def field_index(cfg: Config, name: str, c: int, i: int, j: int, k: int) -> tuple:
    """numpy index of Fortran field(c+1, i, j, k)."""
    nc, lo, *_ = field_extents(cfg, name)
    return (k - lo, j - lo, i - lo, c)
