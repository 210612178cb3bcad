"""Generates the golden fixtures of the particle path by EXECUTING THE
REFERENCE'S OWN FORTRAN SOURCE TEXT.

The reference (MPIEMSES3D) cannot be compiled here: it needs a Fortran
compiler, MPI, HDF5 and FFTW, none of which exist in this image.  Its
particle-path subroutines are, however, plain Fortran 90 over module
arrays, so fortran_subset.py (a small interpreter for exactly the statements
these files use) runs them from the text of

    src/field/grdcrt.F90         grdcrt
    src/pcl2field/psolve2.F90    psolve2
    src/pcl2field/psolve1.F90    psolve1, add_boundary_current(2)
    src/pcl2field/charge.F90     charge, add_boundary_charge
    src/field/rhoupd.F90         rhoupd
    src/pcl/positn.F90           positn
    src/field/bfield.F90         bfield
    src/field/efield.F90         efield
    src/etc/energy.F90           energy (MPI_Reduce of one rank: a no-op)

with IEEE double arithmetic in source order (Python floats: no fused
multiply-add, no reassociation), Fortran integer division and int()
truncation.  What the interpreter does not run is set up here as the
reference's single-rank state would hold it, each item citing its source:

  * module variables: sdoms/sdid/bounds/ctypes/nborps as OhHelp builds them
    for one rank (src/wrapper/ohinit.F90:84-122, ohhelp3.c init_subdomain_*),
    the particle buffer with pbase(1) = 0 and totalp per species;
  * oh3_exchange_borders on one rank (ohhelp3.c set_border_comm): the
    periodic guard copy, restated below in numpy (`exchange`);
  * RANU0 (src/wrapper/wrapper.F90) draws from a fixed list of uniforms,
    the same list the oracle is given;
  * create_simple_collision_boundaries returns an empty list (no internal
    collision boundaries are configured in these cases);
  * logging_debuglog / str are no-ops.

Run from the repository root:

    python tests/golden/make_golden.py [--reference DIR]

It writes tests/golden/<case>.npz; tests/test_golden.py replays every
fixture through the oracle and requires bit-identical results.
"""
from __future__ import annotations

import argparse
import ctypes
import math
import os
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parent.parent))

from fortran_subset import DerivedObj, FArray, Interpreter, parse_source  # noqa: E402

from ctca_b200 import inputs  # noqa: E402
from ctca_b200.emses import INPC, ISPEC, PARTICLE_DTYPE, Body, Config, field_shape  # noqa: E402

SOURCES = ["src/field/grdcrt.F90", "src/pcl2field/psolve2.F90", "src/pcl2field/psolve1.F90",
           "src/pcl2field/charge.F90", "src/field/rhoupd.F90", "src/pcl/positn.F90",
           "src/field/bfield.F90", "src/field/efield.F90", "src/etc/energy.F90"]
# tcs of efield (src/main/inital.F90:78, rescal.F90:132) for the field-step
# fixtures: 2 (c dt)^2 in internal units with c dt / dx = 0.5
TCS = 0.125

# src/main/paramt.F90:44-48
CEB, CAJ, CRH, CRD, CJD, CPH = 1, 2, 3, 4, 5, 6
BNR, CNR = 2, 6
# ctypes of src/wrapper/ohinit.F90:111-122, as ((down), (up)) triples
CTYPES = {CEB: ((0, 0, 2), (-1, -1, 1)), CAJ: ((-1, 2, 3), (-1, -4, 3)), CRH: ((0, 1, 1), (0, -1, 1)),
          CRD: ((0, 1, 1), (0, -1, 1)), CJD: ((-1, 2, 3), (-1, -4, 3)), CPH: ((0, 0, 1), (-1, -1, 1))}


def load_units(ref: Path) -> dict:
    units = {}
    for f in SOURCES:
        units.update(parse_source((ref / f).read_text()))
    return units


# ------------------------------------------------------------ array views
def fview(a: np.ndarray, lo: int, ps_axis: bool = True) -> FArray:
    """Fortran view of an oracle-layout field (nz', ny', nx', nc): the
    reference's (nc, lo:, lo:, lo:[, ps]) with ps extent 1."""
    t = a.transpose(3, 2, 1, 0)
    if ps_axis:
        t = t[..., None]
        return FArray(t, [1, lo, lo, lo, 1])
    return FArray(t, [1, lo, lo, lo])


def fview_sp(a: np.ndarray, lo: int) -> FArray:
    """rhobksp: oracle (nspec, nz', ny', nx', 1) -> (1, lo:, lo:, lo:, ps, is)."""
    t = a.transpose(4, 3, 2, 1, 0)[:, :, :, :, None, :]
    return FArray(t, [1, lo, lo, lo, 1, 1])


def exchange(a: "Field", n, nfbnd, ct) -> None:
    """oh3_exchange_borders for one rank (every neighbour is the rank itself
    on a periodic axis, MPI_PROC_NULL on the others), in place on an
    oracle-layout array whose lower bound is a.lo.  Axis order x, y, z; the
    x exchange spans the inner+upper extents (exti) of y and z, the y
    exchange spans exto of x and exti of z, the z exchange exto of x and y
    (ohhelp3.c set_border_comm and oh3_exchange_borders)."""
    (fl, tl, sl_), (fu, tu, su_) = ct
    lo = a.lo
    ti = [(fl, n[d] + fu + su_ - 1) for d in range(3)]
    to = [(tu, n[d] + tl + sl_ - 1) for d in range(3)]
    arr = a.arr  # (z, y, x, c)
    for d in range(3):
        if nfbnd[d] != 0:
            continue
        rng = []
        for e in range(3):
            if e == d:
                rng.append(None)
            else:
                r0, r1 = to[e] if e < d else ti[e]
                rng.append(slice(r0 - lo, r1 - lo + 1))
        for src0, dst0, sz in ((fl, n[d] + tl, sl_), (n[d] + fu, tu, su_)):
            for s in range(sz):
                si = list(rng)
                di = list(rng)
                si[d] = src0 + s - lo
                di[d] = dst0 + s - lo
                # numpy index order is (z, y, x)
                arr[(di[2], di[1], di[0])] = arr[(si[2], si[1], si[0])].copy()


class Field:
    def __init__(self, arr, lo):
        self.arr = arr
        self.lo = lo


# ------------------------------------------------------------ environment
def single_rank_nborps(cfg: Config) -> np.ndarray:
    """nborps(1:27, ispec, 2) of one rank: the rank itself (0) across
    periodic/reflecting axes, -1 when a crossed axis is absorbing
    (src/etc/nborps.F90 with nodes = 1)."""
    nb = np.zeros((27, ISPEC, 2), dtype=np.int64)
    for nud in range(1, 28):
        off = [(nud - 1) % 3 - 1, ((nud - 1) // 3) % 3 - 1, (nud - 1) // 9 - 1]
        for s in range(cfg.nspec):
            dead = any(off[d] != 0 and cfg.npbnd[s][d] not in (0, 1) for d in range(3))
            nb[nud - 1, s, :] = -1 if dead else 0
    return nb


def make_env(cfg: Config, pbuf: np.ndarray, totalp, f: dict, uniforms: np.ndarray):
    nx, ny, nz, ns = cfg.nx, cfg.ny, cfg.nz, cfg.nspec
    g: dict = {}
    pos = [0]

    def ranu0(dranu, n, icon):
        for i in range(int(n)):
            dranu.data[i] = uniforms[pos[0]]
            pos[0] += 1

    def rann0(*a):
        raise RuntimeError("RANN0 is not reached by these cases")

    def ohhinfo_update(sdom):
        # src/wrapper/ohhinfo.F90:24-48
        s = sdom.data
        g.update(xl=int(s[0, 0]), xu=int(s[1, 0]), yl=int(s[0, 1]), yu=int(s[1, 1]), zl=int(s[0, 2]),
                 zu=int(s[1, 2]))
        g.update(dxl=float(g["xl"]), dxu=float(g["xu"]), dyl=float(g["yl"]), dyu=float(g["yu"]),
                 dzl=float(g["zl"]), dzu=float(g["zu"]))
        g.update(ngx=g["xu"] - g["xl"], ngy=g["yu"] - g["yl"], ngz=g["zu"] - g["zl"])
        g.update(dngx=float(g["ngx"]), dngy=float(g["ngy"]), dngz=float(g["ngz"]))

    def boundaries(*a):
        return DerivedObj(nboundaries=0, destroy=lambda: None)

    ext = {"ranu0": ranu0, "rann0": rann0, "ohhinfo_update": ohhinfo_update,
           "create_simple_collision_boundaries": boundaries,
           "logging_debuglog": lambda *a: None, "str": lambda v: str(v)}

    def arr(vals, dt=np.float64, lb=None):
        a = np.array(vals, dtype=dt)
        return FArray(a, lb)

    sd = np.zeros((2, 3, 1), dtype=np.int64)
    sd[1, :, 0] = (nx, ny, nz)
    bounds = np.zeros((2, 3, 1), dtype=np.int64)
    for d in range(3):
        bounds[:, d, 0] = 1 if cfg.nfbnd[d] == 0 else 2  # bcond, ohinit.F90:86-92
    ct = np.zeros((3, 2, BNR + 1, CNR), dtype=np.int64)
    for c, (down, up) in CTYPES.items():
        for b in range(2):
            ct[:, 0, b, c - 1] = down
            ct[:, 1, b, c - 1] = up
    npb = np.zeros((3, ISPEC), dtype=np.int64)
    q = np.zeros(ISPEC)
    qm = np.zeros(ISPEC)
    for s in range(ns):
        npb[:, s] = list(cfg.npbnd[s])
        q[s] = cfg.q[s]
        qm[s] = cfg.qm[s]
    tp = np.zeros((ISPEC, 2), dtype=np.int64)
    tp[:ns, 0] = totalp
    gc = DerivedObj(influx=FArray(np.zeros((INPC, ISPEC), dtype=np.int64)),
                    infhist=FArray(np.zeros((INPC + 1, INPC, ISPEC), dtype=np.int64), [0, 1, 1]),
                    nesc=FArray(np.zeros((ISPEC + 1) // 2 * 2, dtype=np.int64)),
                    chgacm=FArray(np.zeros((2, INPC))))
    bodies = [cfg.body[i] for i in range(INPC)]
    cyl = np.empty(INPC, dtype=object)
    sph = np.empty(INPC, dtype=object)
    for i, b in enumerate(bodies):
        cyl[i] = DerivedObj(radius=b.radius, align=b.cyl_align, axis=arr(list(b.cyl_axis)),
                            edge=arr(list(b.cyl_edge)))
        sph[i] = DerivedObj(radius=b.radius, center=arr(list(b.sph_center)))
    gco = np.empty(1, dtype=object)
    gco[0] = gc
    lo4 = -4
    g.update({
        "inpc": INPC, "ispec": ISPEC, "ex": 1, "ey": 2, "ez": 3, "bx": 4, "by": 5, "bz": 6, "jx": 1, "jy": 2, "jz": 3,
        "tjx": 7, "tjy": 8, "tjz": 9, "caj": CAJ, "cjd": CJD, "crh": CRH,
        "oh_pcl_alive": 0, "oh_pcl_injected": 1, "oh_pcl_to_be_accumulated": -1,
        "oh_pcl_to_be_accumulated_as_antipcl": -2,
        "pbuf": FArray(pbuf, [1]), "totalp": FArray(tp), "pbase": arr([0, 0], np.int64),
        "nspec": ns, "isse": 1, "npr": FArray(np.zeros(ISPEC, dtype=np.int64)),
        "q": FArray(q), "qm": FArray(qm), "deltaemax": FArray(np.zeros(ISPEC)),
        "pemax": FArray(np.ones(ISPEC)), "mfpath": FArray(np.zeros(ISPEC)),
        "vxyzmax": FArray(np.zeros(ISPEC)), "peth": FArray(np.zeros(ISPEC)), "path": FArray(np.zeros(ISPEC)),
        "vdtx": FArray(np.zeros(ISPEC)), "vdty": FArray(np.zeros(ISPEC)), "vdtz": FArray(np.zeros(ISPEC)),
        "ewmodel": 0, "t": 0.0, "dt": 0.0, "nretard": 0,
        "ew": FArray(np.zeros((2, ISPEC, 1))), "omegaw": FArray(np.zeros(1)),
        "ntch": 0, "rtch": FArray(np.zeros((3, 4))), "e1tch": FArray(np.zeros(4)), "r2cutoff": FArray(np.zeros(4)),
        "xlcol": arr([0.0]), "xucol": arr([0.0]), "ylcol": arr([0.0]), "yucol": arr([0.0]),
        "zlcol": arr([0.0]), "zucol": arr([0.0]),
        "npc": cfg.npc, "line_mode": cfg.line_mode,
        "geotype": arr([b.geotype for b in bodies], np.int64), "ncond": arr([b.ncond for b in bodies], np.int64),
        "sqdscaled": arr([b.sqdscaled for b in bodies]),
        "xlpc": arr([b.xlpc for b in bodies]), "xupc": arr([b.xupc for b in bodies]),
        "ylpc": arr([b.ylpc for b in bodies]), "yupc": arr([b.yupc for b in bodies]),
        "zlpc": arr([b.zlpc for b in bodies]), "zupc": arr([b.zupc for b in bodies]),
        "cylinder": FArray(cyl), "sphere": FArray(sph), "rbowl": -1.0, "rdome": -1.0,
        "slx": float(nx), "sly": float(ny), "slz": float(nz),
        "npbnd": FArray(npb), "nfbnd": FArray(np.array(list(cfg.nfbnd), dtype=np.int64)),
        "nborps": FArray(single_rank_nborps(cfg)),
        "nphgram": FArray(np.zeros((2, ISPEC, 2), dtype=np.int64), [0, 1, 1]),
        "sdid": arr([0, -1], np.int64), "sdoms": FArray(sd), "bounds": FArray(bounds), "ctypes": FArray(ct),
        "gcount": FArray(gco), "dranu": FArray(np.zeros(1)),
        "sey": FArray(np.zeros((INPC, ISPEC))),
        "e0x": cfg.e0[0], "e0y": cfg.e0[1], "e0z": cfg.e0[2],
        "b0x": cfg.b0[0], "b0y": cfg.b0[1], "b0z": cfg.b0[2],
        "zurechole": arr([-1.0]), "boundary_type": "flat-surface", "sfecrrct": 0,
        "eb": fview(f["eb"], -1), "wrk": fview(f["wrk"], lo4, ps_axis=False),
        "aj": fview(f["aj"], lo4), "ajdg": fview(f["ajdg"], lo4),
        "rho": fview(f["rho"], -1), "rhodg": fview(f["rhodg"], -1), "rhobk": fview(f["rhobk"], -1),
        "rhobksp": fview_sp(f["rhobksp"], -1),
        "colf": FArray(np.zeros((1, nx + 9, ny + 9, nz + 9, 1)), [1, lo4, lo4, lo4, 1]),
    })
    ohhinfo_update(FArray(sd[:, :, 0]))
    return g, ext, gc, pos


def counters(gc: DerivedObj) -> dict:
    return {"influx": gc.influx.data.T.astype(np.int32).copy(),          # (ispec, inpc)
            "infhist": gc.infhist.data.transpose(2, 1, 0).astype(np.int32).copy(),  # (ispec, inpc, inpc+1)
            "nesc": gc.nesc.data.astype(np.int32).copy(),
            "chgacm": gc.chgacm.data.T.copy()}                            # (inpc, 2)


# ------------------------------------------------------------ the cases
def base_case(name):
    c = inputs.workload_case(1)
    c.n = (6, 5, 4)
    c.species[0].ppc, c.species[1].ppc = 3, 2
    c.kmax = 2 * np.pi / 4 * 2
    c.seed = 4242
    c.b0 = (0.05, -0.1, 0.2)
    c.e0 = (1e-3, -2e-3, 5e-4)
    return c


def case_defs():
    out = {}
    c = base_case("periodic")
    c.species[0].vth *= 8
    c.species[1].vth *= 30
    out["periodic"] = (c, 1, {"inject": 7, "predead": 4})
    c = base_case("walls")
    c.seed = 4343
    c.species[0].vth *= 16
    c.species[1].vth *= 60
    c.species[0].npbnd = (1, 2, 0)
    c.species[1].npbnd = (2, 1, 1)
    c.nfbnd = (0, 1, 0)
    out["walls"] = (c, 2, {"inject": 5, "predead": 0})
    c = base_case("walls_z")
    c.seed = 4444
    c.species[0].vth *= 16
    c.species[1].vth *= 60
    c.species[0].npbnd = (0, 0, 2)
    c.species[1].npbnd = (0, 0, 1)
    c.nfbnd = (0, 0, 1)
    out["walls_z"] = (c, 1, {"inject": 0, "predead": 0})
    c = base_case("bodies")
    c.seed = 4545
    c.species[0].vth *= 10
    c.species[1].vth *= 40
    c.bodies = [
        dict(geotype=1, ncond=1, xlpc=1.5, xupc=3.0, ylpc=0.5, yupc=2.5, zlpc=0.0, zupc=1.5, sqdscaled=0.7),
        dict(geotype=2, ncond=1, cyl_align=3, cyl_axis=(4.5, 3.5), cyl_edge=(1.0, 3.0), radius=0.8,
             sqdscaled=1.3),
        dict(geotype=3, ncond=0, sph_center=(2.0, 3.5, 2.5), radius=0.9, sqdscaled=0.0),
        dict(geotype=2, ncond=1, cyl_align=1, cyl_axis=(1.0, 3.0), cyl_edge=(3.5, 5.5), radius=0.6,
             sqdscaled=2.0),
        dict(geotype=2, ncond=1, cyl_align=2, cyl_axis=(3.0, 5.0), cyl_edge=(0.0, 2.0), radius=0.7,
             sqdscaled=0.25),
    ]
    out["bodies"] = (c, 1, {"inject": 3, "predead": 2})
    return out


def prepare(c, opts, rng):
    cfg = inputs.make_config(c)
    eb = inputs.make_fields(c)
    p, tp = inputs.make_particles(c)
    p["pid"] = rng.integers(0, 3, p.size)
    # injected particles (preside = OH_PCL_INJECTED) and particles already
    # marked for removal (preside < 0) in each species segment
    base = 0
    for s, t in enumerate(tp):
        seg = np.arange(base, base + int(t))
        pick = rng.choice(seg, opts["inject"] + opts["predead"], replace=False)
        p["preside"][pick[: opts["inject"]]] = 1
        p["preside"][pick[opts["inject"]:]] = -1
        base += int(t)
    return cfg, eb, p, np.array(tp, dtype=np.int64)


def run_case(units, name, c, ustep, opts):
    rng = np.random.default_rng(sum(map(ord, name)))
    cfg, eb, p0, tp = prepare(c, opts, rng)
    uniforms = rng.random(4 * max(1, opts["inject"]) * cfg.nspec + 8)

    def fields():
        f = {nm: np.zeros(field_shape(cfg, nm)) for nm in ("wrk", "aj", "ajdg", "rho", "rhodg", "rhobk", "rhobksp")}
        f["eb"] = eb.copy()
        return f

    out = {"config": np.frombuffer(bytes(cfg), dtype=np.uint8).copy(), "eb": eb.copy(), "pbuf0": p0.copy(),
           "totalp": tp.copy(), "ustep": np.int64(ustep), "uniforms": uniforms.copy()}
    t0 = time.time()
    # grdcrt + psolve2 (velocity/position update with boundary handling)
    f = fields()
    pb = p0.copy()
    g, ext, gc, pos = make_env(cfg, pb, tp, f, uniforms)
    it = Interpreter(units, g, ext)
    it.call("grdcrt", [1])
    out["wrk"] = f["wrk"].copy()
    it.call("psolve2", [1, ustep])
    out["psolve2_pbuf"] = pb.copy()
    out["psolve2_nranu"] = np.int64(pos[0])
    for k, v in counters(gc).items():
        out["psolve2_" + k] = v
    # positn: the position-only advance of the initial state
    f = fields()
    pb = p0.copy()
    g, ext, gc, pos = make_env(cfg, pb, tp, f, uniforms)
    it = Interpreter(units, g, ext)
    it.call("positn", [1, ustep])
    out["positn_pbuf"] = pb.copy()
    out["positn_nranu"] = np.int64(pos[0])
    for k, v in counters(gc).items():
        out["positn_" + k] = v
    # energy of the initial state (kinetic per species and axis)
    g.update(engk=FArray(np.zeros((3, cfg.nspec))), engeb=FArray(np.zeros(2)), cs=1.0,
             rm=FArray(np.array([cfg.rm[i] for i in range(cfg.nspec)], dtype=np.float64)),
             engkg=FArray(np.zeros((3, cfg.nspec))), engebg=FArray(np.zeros(2)), mpi_real8=0, mpi_sum=0, mcw=0)
    ext["mpi_reduce"] = lambda *a: None
    it.call("energy", [])
    out["energy_engk"] = g["engk"].data.copy()
    # grdcrt + psolve1(func=1): zigzag current, then the J border reduction
    f = fields()
    pb = p0.copy()
    g, ext, gc, pos = make_env(cfg, pb, tp, f, uniforms)
    it = Interpreter(units, g, ext)
    it.call("grdcrt", [1])
    it.call("psolve1", [1, ustep, 1])
    out["psolve1_pbuf"] = pb.copy()
    out["psolve1_nranu"] = np.int64(pos[0])
    out["psolve1_aj"] = f["aj"].copy()
    out["psolve1_ajdg"] = f["ajdg"].copy()
    for k, v in counters(gc).items():
        out["psolve1_" + k] = v
    n = (cfg.nx, cfg.ny, cfg.nz)
    exchange(Field(f["aj"], -4), n, list(cfg.nfbnd), CTYPES[CAJ])
    it.call("add_boundary_current", [1])
    out["reduced_aj"] = f["aj"].copy()
    exchange(Field(f["ajdg"], -4), n, list(cfg.nfbnd), CTYPES[CJD])
    it.call("add_boundary_current2", [1])
    out["reduced_ajdg"] = f["ajdg"].copy()
    # charge(func=2) on the pushed particles, some marked for accumulation
    pb2 = pb.copy()
    alive = np.flatnonzero(pb2["nid"] != -1)
    mark = rng.choice(alive, min(6, alive.size), replace=False)
    pb2["preside"][mark[:3]] = -1
    pb2["preside"][mark[3:]] = -2
    out["charge_pbuf_in"] = pb2.copy()
    g["pbuf"] = FArray(pb2, [1])
    it.call("charge", [1, 2])
    out["charge_pbuf"] = pb2.copy()
    for nm in ("rho", "rhodg", "rhobk", "rhobksp"):
        out["charge_" + nm] = f[nm].copy()
    # border reduction of rho (nelem = uelem = 1) and rhodg (uelem = 2*nspec)
    # fsizes(:, :, FRH): -1 .. n+1 on every axis
    fs = FArray(np.array([[-1, n[0] + 1], [-1, n[1] + 1], [-1, n[2] + 1]], dtype=np.int64).T.copy())
    sdom = FArray(g["sdoms"].data[:, :, 0].copy())
    bnd = FArray(g["bounds"].data[:, :, 0].copy())
    ctr = FArray(g["ctypes"].data[:, :, 0, CRH - 1].copy())
    ctd = FArray(g["ctypes"].data[:, :, 0, CRD - 1].copy())
    exchange(Field(f["rho"], -1), n, list(cfg.nfbnd), CTYPES[CRH])
    it.call("add_boundary_charge", [FArray(f["rho"].transpose(3, 2, 1, 0)), 1, 1, sdom, bnd, ctr, fs, 0])
    out["reduced_rho"] = f["rho"].copy()
    nel = f["rhodg"].shape[-1]
    exchange(Field(f["rhodg"], -1), n, list(cfg.nfbnd), CTYPES[CRD])
    it.call("add_boundary_charge", [FArray(f["rhodg"].transpose(3, 2, 1, 0)), nel, 2 * cfg.nspec, sdom, bnd, ctd,
                                    fs, 0])
    out["reduced_rhodg"] = f["rhodg"].copy()
    # rhoupd with the reduced rho and aj
    it.call("rhoupd", [1])
    out["rhoupd_rho"] = f["rho"].copy()
    # the field step around the push: bfield, efield with the reduced aj
    # (no test particles: dlt = 2; no lumped elements), eb border exchange
    g.update(juncan=0, nflag_testp=0, tcs=TCS, ngap=0, mode_dipole=0)
    it.call("bfield", [1])
    out["bfield_eb"] = f["eb"].copy()
    it.call("efield", [1])
    out["efield_eb"] = f["eb"].copy()
    exchange(Field(f["eb"], -1), n, list(cfg.nfbnd), CTYPES[CEB])
    out["exchange_eb"] = f["eb"].copy()
    out["tcs"] = np.float64(TCS)
    print(f"{name}: {p0.size} particles, {time.time() - t0:.1f} s", flush=True)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("EMSES_REFERENCE", str(HERE.parents[2] / "reference")),
                    help="the reference source tree ($EMSES_REFERENCE, else a `reference` directory beside "
                         "this repository)")
    ap.add_argument("--only", default=None)
    a = ap.parse_args()
    units = load_units(Path(a.reference))
    for name, (c, ustep, opts) in case_defs().items():
        if a.only and name != a.only:
            continue
        out = run_case(units, name, c, ustep, opts)
        np.savez_compressed(HERE / f"{name}.npz", **out)


if __name__ == "__main__":
    main()
