"""Golden vectors of the injection supervisors, made by EXECUTING THE
REFERENCE'S OWN FORTRAN SOURCE TEXT (fortran_subset.py, as make_golden.py
does for the particle path).

psuper2.F90 as a whole uses statements the small interpreter does not run
(print, array sections, the OhHelp mapping calls of the inner-boundary
branch), so the pieces on this path are cut out of the file verbatim and
run on their own:

  * the six outer-boundary inflow blocks (x-bottom .. z-top,
    src/pcl/psuper2.F90:114-292), wrapped in a subroutine whose variables
    are the module state the blocks read;
  * the rectangular-plane emission dispatch on nemd (psuper2.F90:333-362)
    and the contained emit_from_rectangular_surf (:554-576) it calls;
  * the emission count of psuper3 (psuper3.F90:68-69), over a grid of
    steps and fluxes;
  * the emission pairs of psuper3 (emit_from_rectangle, psuper3.F90:142-208,
    with its own emit_from_rectangular_surf, :210-240; the BLOCK construct
    around three local declarations is unwrapped), oh3_map_particle_to_
    subdomain answering this rank.

RANU0 hands out a fixed list of uniforms; oh2_inject_particle collects the
records.  The fixture holds the tables, the uniforms each piece consumed,
the counts and the records; tests/test_golden_supervisors.py checks
ctca_b200/inject.py (and so, through the device tests, the device
supervisors) against it.

Run from the repository root:

    python tests/golden/make_golden_supervisors.py [--reference DIR]
"""
from __future__ import annotations

import argparse
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parent.parent))

from fortran_subset import DerivedObj, FArray, Interpreter, parse_source  # noqa: E402

from ctca_b200 import tables  # noqa: E402
from ctca_b200.emses import PARTICLE_DTYPE  # noqa: E402

FIELDS = ("x", "y", "z", "vx", "vy", "vz", "pid", "preside", "nid", "spec")


def cut(lines, start_pat, stop_pat, include_stop=False):
    """Lines from the first one containing start_pat up to the first later
    one containing stop_pat."""
    i0 = next(i for i, l in enumerate(lines) if start_pat in l)
    i1 = next(i for i in range(i0 + 1, len(lines)) if stop_pat in lines[i])
    return lines[i0:i1 + (1 if include_stop else 0)]


def pieces(ref: Path) -> str:
    lines = (ref / "src/pcl/psuper2.F90").read_text().splitlines()
    inflow = cut(lines, "!-------------------- x-bottom", "!============================== from inner boundary")
    assert any("narrzb(is)" in l for l in inflow) and sum("oh2_inject_particle" in l for l in inflow) == 6
    # the dispatch on nemd of the rectangular surfaces, up to its end if
    i0 = next(i for i, l in enumerate(lines) if "if(nemd(iepl).eq. 1) then" in l)
    i1 = next(i for i in range(i0, len(lines)) if lines[i].strip() == "end if")
    emit = lines[i0:i1 + 1]
    assert sum("call emit_from_rectangular_surf" in l for l in emit) == 6
    surf = cut(lines, "subroutine emit_from_rectangular_surf &", "end subroutine emit_from_rectangular_surf",
               include_stop=True)
    text = ["subroutine golden_inflow(ustep)",
            "  integer(kind=4) :: m, iran, addr1, addr2, icon, ustep"] + inflow + [
            "end subroutine golden_inflow", "",
            "subroutine golden_emit(m)",
            "  integer(kind=4) :: m"] + emit + ["end subroutine golden_emit", ""] + surf
    return "\n".join(text) + "\n"


def pieces3(ref: Path) -> str:
    lines = (ref / "src/pcl/psuper3.F90").read_text().splitlines()
    rect = cut(lines, "subroutine emit_from_rectangle", "end subroutine", include_stop=True)
    rect[0] = rect[0].replace("subroutine emit_from_rectangle", "subroutine emit_from_rectangle()")  # empty list
    surf = cut(lines, "subroutine emit_from_rectangular_surf(", "end subroutine emit_from_rectangular_surf",
               include_stop=True)
    surf = [l for l in surf if not (l.strip().startswith("block") or l.strip().startswith("end block"))]
    assert sum("oh2_inject_particle" in l for l in rect) == 2
    return "\n".join(rect + [""] + surf) + "\n"


def record_of(p) -> tuple:
    return tuple(p[f] for f in FIELDS)


def make(ref: Path) -> dict:
    units = parse_source(pieces(ref))
    rng = np.random.default_rng(20251203)
    npr = 64
    ext = (24, 20, 32)
    uniforms = rng.random(200000)
    pos = [0]
    injected = []

    def ranu0(dranu, n, icon):
        for i in range(int(n)):
            dranu.data[i] = uniforms[pos[0]]
            pos[0] += 1

    def inject_rec(p):
        injected.append(record_of(p))

    tab = lambda a: FArray(np.asarray(a, dtype=np.float64).copy(), [1])  # noqa: E731
    # tables of one species (nprs = 1): normal speeds per face, tangential ones
    # (the reference's own table builders, ctca_b200/tables.py, pinned by
    # make_golden_tables.py)
    vth, vd = 0.05, 0.02
    stream = tables.Ranu0(900)
    built = tables.inflow_tables(npr, 1, (vd, -vd, 0.0), vth, vth, stream)
    t = {k: built[k] for k in ("vxf", "vxb", "vyf", "vyb", "vzf", "vzb", "vxr", "vyr", "vzr")}
    ustep, injct, istep, lstep = 2, 1, 7, 0
    arr = {"arrxf": 13.7, "arrxb": 9.2, "arryf": 11.4, "arryb": 8.9, "arrzf": 15.3, "arrzb": 12.1}
    zssurf = 0.004  # some z-bottom particles stay below: dropped (psuper2.F90 `cycle`)
    pinj = FArray(np.zeros(1, dtype=PARTICLE_DTYPE), [1])
    g = {"is": 1, "nprs": 1, "npr": FArray(np.array([npr], dtype=np.int64), [1]),
         "npbnd": FArray(np.full((3, 1), 2, dtype=np.int64), [1, 1]),
         "bared": FArray(np.ones((2, 3, 1), dtype=np.int64), [1, 1, 1]),
         "sdid": FArray(np.array([0], dtype=np.int64), [1]),
         "istep": istep, "lstep": lstep, "injct": FArray(np.array([injct], dtype=np.int64), [1]),
         "injctisw": FArray(np.array([injct * ustep], dtype=np.int64), [1]),
         "xl": 0, "xu": ext[0], "yl": 0, "yu": ext[1], "zl": 0, "zu": ext[2],
         "zssurf": zssurf, "ubhole": -1.0e30, "dranu": FArray(np.zeros(200000), [1]), "pinj": pinj}
    for k, v in t.items():
        g[k] = tab(v)
    for k, v in arr.items():
        g[k] = FArray(np.array([v]), [1])
        g["n" + k] = FArray(np.zeros(1, dtype=np.int64), [1])
    it = Interpreter(units, g, {"ranu0": ranu0, "oh2_inject_particle": inject_rec})
    it.call("golden_inflow", [ustep])
    out = {"npr": np.int64(npr), "ext": np.array(ext, dtype=np.int64), "ustep": np.int64(ustep),
           "injct": np.int64(injct), "istep": np.int64(istep), "lstep": np.int64(lstep), "zssurf": np.float64(zssurf),
           "uniforms": uniforms[:pos[0]].copy(), "inflow_records": np.array(injected, dtype=PARTICLE_DTYPE)}
    for k, v in t.items():
        out["tab_" + k] = v
    for k in arr:
        out["arr_" + k] = np.float64(arr[k])
        out["count_" + k] = np.int64(g["n" + k].data[0])
    used_inflow = pos[0]
    # plane emission: per face, n particles with RANU0(dranu, n*6) first
    em = tables.emission_tables(npr, npr, 0.0, 0.01, 0.01, 0.0, stream)
    vnormf, vtangf = em["vnormf"], em["vtangf"]
    g.update(vnormf=tab(vnormf), vtangf=tab(vtangf), iepl=1)
    faces = [(1, 16.0), (-1, 8.0), (2, 12.5), (-2, 7.0), (3, 18.0), (-3, 14.0)]
    bounds = {"xl": 4.0, "xu": 20.0, "yl": 3.0, "yu": 17.0, "zl": 6.0, "zu": 26.0}
    emitted = []
    for nemd, grd in faces:
        n = 40
        g["nemd"] = FArray(np.array([nemd], dtype=np.int64), [1])
        g["peject"] = FArray(np.array([DerivedObj(grd=grd, **bounds)], dtype=object), [1])
        ranu0(g["dranu"], n * 6, 0)
        for m in range(1, n + 1):
            pinj.data[0] = np.zeros(1, dtype=PARTICLE_DTYPE)[0]
            it.call("golden_emit", [m])
            emitted.append(record_of(pinj.data[0]))
    out["emit_faces"] = np.array(faces, dtype=np.float64)
    out["emit_bounds"] = np.array([bounds[k] for k in ("xl", "xu", "yl", "yu", "zl", "zu")])
    out["emit_n"] = np.int64(40)
    out["emit_uniforms"] = uniforms[used_inflow:pos[0]].copy()
    out["emit_vnormf"] = vnormf
    out["emit_vtangf"] = vtangf
    out["emit_records"] = np.array(emitted, dtype=PARTICLE_DTYPE)
    # psuper3 emission pairs: nemit(iepl) pairs per face
    used_plane = pos[0]
    units3 = parse_source(pieces3(ref))
    pinj2 = FArray(np.zeros(2, dtype=PARTICLE_DTYPE), [1])
    injected.clear()
    g3 = dict(g)
    g3.update(pinj=pinj2, m=0, xl=0, xu=ext[0], yl=0, yu=ext[1], zl=0, zu=ext[2])
    it3 = Interpreter(units3, g3, {"ranu0": ranu0, "oh2_inject_particle": inject_rec,
                                   "oh3_map_particle_to_subdomain": lambda *a: 0})
    for nemd, grd in faces:
        g3["nemd"] = FArray(np.array([nemd], dtype=np.int64), [1])
        g3["nemit"] = FArray(np.array([40], dtype=np.int64), [1])
        g3["peject"] = FArray(np.array([DerivedObj(grd=grd, **bounds)], dtype=object), [1])
        ranu0(g3["dranu"], 40 * 6, 0)
        it3.call("emit_from_rectangle", [])
    out["pair_uniforms"] = uniforms[used_plane:pos[0]].copy()
    # the emission count statement, cut out of psuper3.F90
    lines = (ref / "src/pcl/psuper3.F90").read_text().splitlines()
    cnt = cut(lines, "nemit(iepl) = (int((istep + lstep)*fluxf(iepl), 8)", "ipcplane = ipcpl(iepl)")
    units_c = parse_source("\n".join(["subroutine golden_count(ustep)", "  integer(kind=4) :: ustep"] + cnt +
                                     ["end subroutine golden_count", ""]))
    rows = []
    for istep in (0, 1, 7, 123):
        for lstep in (0, 5):
            for injct in (1, 3):
                for fluxf in (0.37, 2.5, 1048576.0, 13.09):
                    for ustep in (1, 2):
                        gc = {"istep": istep, "lstep": lstep, "iepl": 1, "is": 1,
                              "injct": FArray(np.array([injct], dtype=np.int64), [1]),
                              "fluxf": FArray(np.array([fluxf]), [1]),
                              "nemit": FArray(np.zeros(1, dtype=np.int64), [1])}
                        Interpreter(units_c, gc, {}).call("golden_count", [ustep])
                        rows.append((istep, lstep, injct, fluxf, ustep, int(gc["nemit"].data[0])))
    out["count_rows"] = np.array(rows, dtype=np.float64)
    out["pair_records"] = np.array(injected, dtype=PARTICLE_DTYPE)
    cylinder_emission(ref, out)
    psuper1_current(ref, out)
    return out


def psuper1_current(ref: Path, out: dict) -> None:
    """psuper1's six outer-face inflow blocks (psuper1.F90:120-323) and the
    contained current_deposition (:859-988) it calls after each injected
    particle, cut out verbatim and run on one species: the records and the
    zigzag current of their paths into the domain (wrk(TJX:TJZ))."""
    lines = (ref / "src/pcl/psuper1.F90").read_text().splitlines()
    blocks = cut(lines, "! x-bottom", "!============================== from inner boundary")
    assert sum("call current_deposition" in l for l in blocks) == 6
    dep = cut(lines, "subroutine current_deposition", "end subroutine current_deposition", include_stop=True)
    text = ["subroutine golden_psuper1(ustep)",
            "  integer(kind=4) :: m, iran, addr1, addr2, icon, ustep"] + blocks + [
            "end subroutine golden_psuper1", ""] + dep
    units = parse_source("\n".join(text) + "\n")
    rng = np.random.default_rng(20251205)
    npr = 64
    ext = (16, 12, 20)
    ustep, injct, istep, lstep = 2, 1, 5, 0
    stream = tables.Ranu0(902)
    built = tables.inflow_tables(npr, 1, (0.01, -0.02, 0.0), 0.05, 0.05, stream)
    uniforms = rng.random(100000)
    pos = [0]
    injected = []

    def ranu0(dranu, n, icon):
        dranu.data[:int(n)] = uniforms[pos[0]:pos[0] + int(n)]
        pos[0] += int(n)

    tab = lambda a: FArray(np.asarray(a, dtype=np.float64).copy(), [1])  # noqa: E731
    arr = {"arrxf": 7.3, "arrxb": 5.2, "arryf": 6.4, "arryb": 4.9, "arrzf": 8.3, "arrzb": 6.1}
    g = {"is": 1, "nprs": 1, "npr": FArray(np.array([npr], dtype=np.int64), [1]),
         "npbnd": FArray(np.full((3, 1), 2, dtype=np.int64), [1, 1]),
         "bared": FArray(np.ones((2, 3, 1), dtype=np.int64), [1, 1, 1]),
         "sdid": FArray(np.array([0], dtype=np.int64), [1]),
         "istep": istep, "lstep": lstep, "injct": FArray(np.array([injct], dtype=np.int64), [1]),
         "injctisw": FArray(np.array([injct * ustep], dtype=np.int64), [1]),
         "xl": 0, "xu": ext[0], "yl": 0, "yu": ext[1], "zl": 0, "zu": ext[2],
         "zssurf": -1.0e30, "ubhole": -1.0e30, "dranu": FArray(np.zeros(100000), [1]),
         "pinj": FArray(np.zeros(1, dtype=PARTICLE_DTYPE), [1]), "rustep": 1.0 / ustep,
         "tjx": 7, "tjy": 8, "tjz": 9,
         "wrk": FArray(np.zeros((9, ext[0] + 9, ext[1] + 9, ext[2] + 9)), [1, -4, -4, -4])}
    for k in ("xlocalb", "ylocalb", "zlocalb", "xb", "yb", "zb", "xlocala", "ylocala", "zlocala", "xa", "ya", "za",
              "xr", "yr", "zr", "xd1", "yd1", "zd1", "xd2", "yd2", "zd2", "vvx1", "vvy1", "vvz1", "vvx2", "vvy2",
              "vvz2"):
        g[k] = 0.0
    for s_ in ("1", "2"):
        for c in "xyz":
            for w in "1234":
                g[f"v{c}{s_}w{w}"] = 0.0
    for k in ("ib", "jb", "kb", "i1b", "j1b", "k1b", "ia", "ja", "ka", "i1a", "j1a", "k1a"):
        g[k] = 0
    types = {k: ("integer" if isinstance(v, int) else "real") for k, v in g.items() if isinstance(v, (int, float))}
    t = {k: built[k] for k in ("vxf", "vxb", "vyf", "vyb", "vzf", "vzb", "vxr", "vyr", "vzr")}
    for k, v in t.items():
        g[k] = tab(v)
    for k, v in arr.items():
        g[k] = FArray(np.array([v]), [1])
        g["n" + k] = FArray(np.zeros(1, dtype=np.int64), [1])
    Interpreter(units, g, {"ranu0": ranu0, "oh2_inject_particle": lambda p: injected.append(record_of(p))},
                types).call("golden_psuper1", [ustep])
    out["p1_ext"] = np.array(ext, dtype=np.int64)
    out["p1_setup"] = np.array([npr, ustep, injct, istep, lstep], dtype=np.int64)
    for k, v in t.items():
        out["p1_tab_" + k] = v
    for k in arr:
        out["p1_arr_" + k] = np.float64(arr[k])
        out["p1_count_" + k] = np.int64(g["n" + k].data[0])
    out["p1_uniforms"] = uniforms[:pos[0]].copy()
    out["p1_records"] = np.array(injected, dtype=PARTICLE_DTYPE)
    out["p1_wrk"] = g["wrk"].data[6:9].copy()  # TJX..TJZ, (3, nx + 9, ny + 9, nz + 9)


# (align, radius, omni, ncond, nemd, grd): the end caps and the three kinds of
# side surface of cylinders along x, y and z
CYL_CASES = [(3, 4.5, 0, 0, 3, 20.0), (3, 4.5, 0, 0, -3, 6.0), (3, 4.5, 0, 0, 1, 0.0), (3, 0.6, 0, 0, -2, 0.0),
             (3, 4.5, 1, 1, 2, 0.0), (1, 3.0, 0, 0, 1, 15.0), (1, 3.0, 0, 0, 2, 0.0), (1, 0.4, 0, 0, -3, 0.0),
             (2, 2.5, 0, 0, -2, 4.0), (2, 2.5, 0, 0, 3, 0.0), (2, 2.5, 1, 0, 1, 0.0)]
CYL_AXIS = (12.0, 10.5)
CYL_BOUNDS = {"xl": 4.0, "xu": 20.0, "yl": 3.0, "yu": 17.0, "zl": 6.0, "zu": 26.0}
CYL_PSI = {"psixy": 0.3, "psizx": 1.1, "psizy": 2.0}
CYL_N = 24


def pieces_cyl(ref: Path) -> str:
    lines = (ref / "src/pcl/psuper3.F90").read_text().splitlines()
    cyl = cut(lines, "subroutine emit_from_cylinder", "end subroutine", include_stop=True)
    cyl[0] = cyl[0].replace("subroutine emit_from_cylinder", "subroutine emit_from_cylinder()")  # empty list
    assert sum("oh2_inject_particle" in l for l in cyl) == 4
    text = cyl + [""]
    for name in ("emit_from_circular_surf", "emit_from_cylindrical_surf1", "emit_from_cylindrical_surf2",
                 "emit_from_cylindrical_surf3"):
        text += cut(lines, f"subroutine {name}(", f"end subroutine {name}", include_stop=True) + [""]
    return "\n".join(text) + "\n"


def cylinder_emission(ref: Path, out: dict) -> None:
    """psuper3's emission from cylinders (emit_from_cylinder and the four
    surface routines it calls, psuper3.F90:241-528) cut out verbatim and run
    per case: 6n uniforms from a fixed generator, the reference's emission
    tables of one species (ctca_b200.tables, pinned by make_golden_tables.py)."""
    units = parse_source(pieces_cyl(ref))
    npr = 64
    tb = tables.emission_tables(npr, npr, 0.0, 0.01, 0.01, 0.0, tables.Ranu0(901))
    rng = np.random.default_rng(20251204)
    injected = []
    pinj = FArray(np.zeros(2, dtype=PARTICLE_DTYPE), [1])
    tab = lambda a: FArray(np.asarray(a, dtype=np.float64).copy(), [1])  # noqa: E731
    g = {"is": 1, "nprs": 1, "npr": FArray(np.array([npr], dtype=np.int64), [1]), "m": 0, "iepl": 1, "ipcplane": 1,
         "ipc": 1, "omni": 0, "align": 0.0, "radius": 0.0, "pi2": float(np.arccos(-1.0)) * 2.0,
         "sdid": FArray(np.array([0], dtype=np.int64), [1]), "pinj": pinj,
         "xl": 0, "xu": 32, "yl": 0, "yu": 32, "zl": 0, "zu": 32, "dranu": FArray(np.zeros(6 * CYL_N), [1])}
    g.update(CYL_PSI)
    for k in ("vnormf", "vtangf", "runiform", "vnormc", "vtangc", "psicos"):
        g[k] = tab(tb[k])
    types = {"align": "real", "radius": "real", "m": "integer", "omni": "integer"}
    it = Interpreter(units, g, {"oh2_inject_particle": lambda p: injected.append(record_of(p)),
                                "oh3_map_particle_to_subdomain": lambda *a: 0}, types)
    uni = []
    for align, radius, omni, ncond, nemd, grd in CYL_CASES:
        u = rng.random(6 * CYL_N)
        uni.append(u)
        g["dranu"].data[:] = u
        g["omni"] = omni
        g["ncond"] = FArray(np.array([ncond], dtype=np.int64), [1])
        g["nemd"] = FArray(np.array([nemd], dtype=np.int64), [1])
        g["nemit"] = FArray(np.array([CYL_N], dtype=np.int64), [1])
        g["cylinder"] = FArray(np.array([DerivedObj(align=align, radius=radius,
                                                    axis=FArray(np.array(CYL_AXIS), [1]))], dtype=object), [1])
        g["peject"] = FArray(np.array([DerivedObj(grd=grd, **CYL_BOUNDS)], dtype=object), [1])
        it.call("emit_from_cylinder", [])
    out["cyl_cases"] = np.array(CYL_CASES, dtype=np.float64)
    out["cyl_axis"] = np.array(CYL_AXIS)
    out["cyl_bounds"] = np.array([CYL_BOUNDS[k] for k in ("xl", "xu", "yl", "yu", "zl", "zu")])
    out["cyl_psi"] = np.array([CYL_PSI[k] for k in ("psixy", "psizx", "psizy")])
    out["cyl_n"] = np.int64(CYL_N)
    out["cyl_uniforms"] = np.concatenate(uni)
    for k in ("vnormf", "vtangf", "runiform", "vnormc", "vtangc", "psicos"):
        out["cyl_" + k] = tb[k]
    out["cyl_records"] = np.array(injected, dtype=PARTICLE_DTYPE)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("EMSES_REFERENCE", str(HERE.parents[2] / "reference")),
                    help="the reference source tree ($EMSES_REFERENCE, else a `reference` directory beside "
                         "this repository)")
    args = ap.parse_args()
    out = make(Path(args.reference))
    np.savez_compressed(HERE / "supervisors.npz", **out)
    print(f"inflow records {out['inflow_records'].size}, emitted {out['emit_records'].size}, "
          f"pair records {out['pair_records'].size}")


if __name__ == "__main__":
    main()
