"""Golden vectors of the reference's velocity tables, made by EXECUTING THE
REFERENCE'S OWN FORTRAN SOURCE TEXT (fortran_subset.py) with the reference's
own random stream.

Pieces cut verbatim out of the reference tree and run:

  * src/etc/lemses.F90: vflux, vinit, ringds, rexch, arange, arymod;
  * src/wrapper/wrapper.F90: drann0l (the RANN0 of the table code);
  * src/main/inipin.F90: the tables of the open outer boundaries (the
    `nflag_emit(is) .eq. 0` branch of the second species loop, from its IF
    to its CYCLE, closed with END IF and wrapped in the species loop with
    the loop's first four statements), and the contained subroutine
    assign_velocity (the emission tables).

RANU0 / DRANU0 / DRANU0L hand out the reference's Mersenne Twister stream:
init_genrand(seed) and genrand_res53 of lib/mtarm/mt19937arm.c, compiled
into oracle/_ref by oracle/Makefile and read through oracle.ranu0_stream.
The fixture holds the first draws of that stream (which pin
ctca_b200.tables.Ranu0) and every table; tests/test_golden_tables.py
checks ctca_b200/tables.py against it bit for bit.

Run from the repository root (after `make -C oracle`):

    python tests/golden/make_golden_tables.py [--reference DIR]
"""
from __future__ import annotations

import argparse
import os
import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parents[1]))

from fortran_subset import FArray, Interpreter, parse_source  # noqa: E402

from oracle import oracle as O  # noqa: E402

STREAM_PIN = 4096


def cut_unit(text: str, kind: str, name: str) -> str:
    """The text of one unit, from its header to the first END of its kind
    (named or not: contained units of the reference end with a bare END
    SUBROUTINE)."""
    m = re.search(r"^[ \t]*%s\s+%s\b.*?^[ \t]*end\s+%s\b[^\n]*\n" % (kind, name, kind), text,
                  re.S | re.M | re.I)
    if not m:
        raise SystemExit(f"{kind} {name} not found")
    return m.group(0)


class Stream:
    """The reference's RANU0: its own MT19937 (oracle/_ref), served in order."""

    def __init__(self, seed: int, n: int = 3_000_000):
        self.u = O.ranu0_stream(seed, n)
        self.k = 0

    def take(self, n):
        n = int(n)
        if self.k + n > self.u.size:
            raise SystemExit("stream too short")
        r = self.u[self.k:self.k + n]
        self.k += n
        return r

    def externals(self):
        def ranu0(arr, n, icon, *rest):
            arr.data[:int(n)] = self.take(n)
        return {"ranu0": ranu0, "dranu0": ranu0, "dranu0l": ranu0}


def lemses_units(ref: Path) -> dict:
    lem = (ref / "src/etc/lemses.F90").read_text()
    wrp = (ref / "src/wrapper/wrapper.F90").read_text()
    text = "\n".join(cut_unit(lem, "subroutine", n) for n in ("vflux", "vinit", "ringds", "rexch", "arange",
                                                              "arymod"))
    text += "\n" + cut_unit(wrp, "subroutine", "drann0l")
    units = parse_source(text)
    units["rann0"] = units["drann0l"]  # the generic RANN0 on an integer(8) count
    return units


def run_builders(units: dict, out: dict) -> None:
    """The table builders on their own, a fresh stream (seed) per case."""
    def call(name, args, seed):
        st = Stream(seed, 200_000)
        it = Interpreter(units, {}, st.externals())
        it.call(name, args)
        return it.last_frame, st.k

    vf = [(1000, 0.0, 1.0, 1), (1000, 0.3, 1.0, 1), (1000, 0.3, 1.0, -1), (777, 0.5, 0.2, -1),
          (512, 0.05, 0.2, 1), (640, 2.0, 0.5, -1), (300, 1.0e-3, 0.01, 1)]
    rows = []
    for c, (na, v0, vt, isl) in enumerate(vf):
        ar = FArray(np.zeros(na))
        fr, used = call("vflux", [ar, na, v0, vt, isl, 0], 100 + c)
        out[f"vflux_{c}"] = ar.data.copy()
        rows.append((na, v0, vt, isl, 100 + c, fr.vars["icon"], used))
    out["vflux_cases"] = np.array(rows, dtype=np.float64)
    vi = [(1000, 0.1, 0.5, 0.0), (999, 0.0, 1.0, 0.0), (800, 0.2, 0.0, 2.0), (800, 0.0, 0.3, -1.5),
          (400, 0.05, 0.0, 0.5)]
    rows = []
    for c, (na, v0, vt, xlos) in enumerate(vi):
        ar = FArray(np.zeros(na))
        fr, used = call("vinit", [ar, na, v0, vt, xlos], 200 + c)
        out[f"vinit_{c}"] = ar.data.copy()
        rows.append((na, v0, vt, xlos, 200 + c, fr.vars["v0"], fr.vars["vt"], used))
    out["vinit_cases"] = np.array(rows, dtype=np.float64)
    rg = [(600, 1.0, 0.5), (500, 0.05, 0.1)]
    rows = []
    for c, (na, vt, bbb) in enumerate(rg):
        ar = FArray(np.zeros(na))
        fr, used = call("ringds", [ar, na, vt, bbb], 300 + c)
        out[f"ringds_{c}"] = ar.data.copy()
        rows.append((na, vt, bbb, 300 + c, used))
    out["ringds_cases"] = np.array(rows, dtype=np.float64)
    rn = [(0.0, 1.0, 1), (0.5, 0.2, 1000), (-0.1, 0.03, 999)]
    rows = []
    for c, (am, sd, n) in enumerate(rn):
        ar = FArray(np.zeros(n))
        fr, used = call("rann0", [am, sd, ar, n, 0], 400 + c)
        out[f"rann0_{c}"] = ar.data.copy()
        rows.append((am, sd, n, 400 + c, used))
    out["rann0_cases"] = np.array(rows, dtype=np.float64)
    # rexch of several arrays at once (the same pairs in each)
    n = 333
    i1 = FArray(np.arange(1, n + 1, dtype=np.int64))
    d1 = FArray(np.arange(n, dtype=np.float64) * 0.5)
    d2 = FArray(-np.arange(n, dtype=np.float64))
    st = Stream(500, 10_000)
    Interpreter(units, {}, st.externals()).call("rexch", [n], kw={"i1": i1, "d1": d1, "d5": d2})
    out["rexch_i1"], out["rexch_d1"], out["rexch_d5"] = i1.data.copy(), d1.data.copy(), d2.data.copy()
    out["rexch_case"] = np.array([n, 500, st.k], dtype=np.float64)


INFLOW_SPECIES = {  # two species, the second with nphi = 2 (arymod spreads its tables)
    "npr": [1000, 600], "nphi": [1, 2], "vdtx": [0.1, -0.2], "vdty": [-0.05, 0.0], "vdtz": [0.0, 0.3],
    "peth": [1.0, 0.3], "path": [0.8, 0.3], "npin": [32768.0, 32768.0],
}
INFLOW_GRID = {"slx": 32.0, "sly": 32.0, "slz": 24.0, "xl": 0.0, "xu": 32.0, "yl": 0.0, "yu": 32.0, "zl": 0.0,
               "zu": 24.0, "dt": 0.5, "mltstp": 1}


def run_inflow(ref: Path, units: dict, out: dict, seed: int = 600) -> None:
    ip = (ref / "src/main/inipin.F90").read_text().splitlines()
    a = next(i for i, l in enumerate(ip) if re.match(r"\s*if \(\(nflag_emit\(is\) \.eq\. 0\) \.and\. &", l))
    b = next(i for i in range(a, len(ip)) if ip[i].strip() == "cycle")
    head = next(i for i, l in enumerate(ip) if re.match(r"\s*ISL2: do is = 1, nspec", l))
    body = "\n".join(ip[head + 1:head + 5]) + "\n" + "\n".join(ip[a:b]) + "\nend if\n"
    text = "subroutine golden_inflow()\ndo is = 1, nspec\n" + body + "end do\nend subroutine golden_inflow\n"
    u = dict(units)
    u.update(parse_source(text))
    sp = INFLOW_SPECIES
    ns = len(sp["npr"])
    tot = sum(sp["npr"])

    def arr(v, dt=np.float64):
        return FArray(np.array(v, dtype=dt))
    g = {"nspec": ns, "myid": 0, "nee": 0, "ns": 0, "ne": 0, "is": 0, "iconf": 0, "iconb": 0, "icon": 0,
         "pdf": 0.0, "pdb": 0.0, "aa": 0.0, "bb": 0.0, "pi": float(np.arccos(-1.0)),
         "nflag_emit": arr([0] * ns, np.int64), "npbnd": FArray(np.full((3, ns), 2, dtype=np.int64)),
         "npr": arr(sp["npr"], np.int64), "nphi": arr(sp["nphi"], np.int64), "npq": arr([0] * ns, np.int64),
         "vdtx": arr(sp["vdtx"]), "vdty": arr(sp["vdty"]), "vdtz": arr(sp["vdtz"]), "peth": arr(sp["peth"]),
         "path": arr(sp["path"]), "npin": arr(sp["npin"]), "injct": arr([1] * ns, np.int64),
         "inpf": arr([1] * ns, np.int64), "inpb": arr([1] * ns, np.int64)}
    for k in ("arrxf", "arrxb", "arryf", "arryb", "arrzf", "arrzb"):
        g[k] = arr([0.0] * ns)
    for k in ("vxf", "vyf", "vzf", "vxb", "vyb", "vzb", "vxr", "vyr", "vzr"):
        g[k] = arr([0.0] * tot)
    g.update(INFLOW_GRID)
    types = {k: "integer" for k in ("nspec", "myid", "nee", "ns", "ne", "is", "iconf", "iconb", "icon",
                                    "mltstp")}
    types.update({k: "real" for k in ("pdf", "pdb", "aa", "bb", "pi", "slx", "sly", "slz", "xl", "xu", "yl", "yu",
                                      "zl", "zu", "dt")})
    st = Stream(seed)
    Interpreter(u, g, st.externals(), types).call("golden_inflow", [])
    for k in ("vxf", "vyf", "vzf", "vxb", "vyb", "vzb", "vxr", "vyr", "vzr", "arrxf", "arrxb", "arryf", "arryb",
              "arrzf", "arrzb"):
        out[f"inflow_{k}"] = g[k].data.copy()
    out["inflow_case"] = np.array([seed, st.k], dtype=np.float64)
    out["inflow_species"] = np.array([[sp[k][s] for k in ("npr", "nphi", "vdtx", "vdty", "vdtz", "peth", "path",
                                                           "npin")] for s in range(ns)], dtype=np.float64)
    gr = INFLOW_GRID
    out["inflow_grid"] = np.array([gr["slx"], gr["sly"], gr["slz"], gr["xu"] - gr["xl"], gr["yu"] - gr["yl"],
                                   gr["zu"] - gr["zl"], gr["dt"]], dtype=np.float64)


EMIT_SPECIES = {"npr": [800, 500], "nphi": [1, 2], "spa": [0.0, 0.1], "abvdem": [0.0, 0.05], "spe": [0.0, 0.02],
                "peth": [0.01, 0.2], "path": [0.01, 0.3]}


def run_emission(ref: Path, units: dict, out: dict, variant: int, seed: int) -> None:
    """assign_velocity for both species; variant 1 adds the second
    populations (path(nspec+1), peth(nspec+1), mainprop)."""
    ip = (ref / "src/main/inipin.F90").read_text()
    text = cut_unit(ip, "subroutine", "assign_velocity")
    u = dict(units)
    u.update(parse_source(text))
    sp = EMIT_SPECIES
    ns = len(sp["npr"])
    tot = sum(sp["npr"])

    def arr(v, dt=np.float64):
        return FArray(np.array(v, dtype=dt))
    path2, peth2 = (0.5, 0.2) if variant else (0.0, 0.0)
    g = {"nspec": ns, "is": 0, "ns": 0, "m": 0, "iconf": 0, "icon": 0, "nprfrac1": 0, "nprfrac2": 0,
         "mainprop": 0.7, "pi": float(np.arccos(-1.0)), "psi1": 0.0, "psi2": 0.0,
         "npr": arr(sp["npr"], np.int64), "npq": arr([n // p for n, p in zip(sp["npr"], sp["nphi"])], np.int64),
         "inpf": arr([1] * ns, np.int64), "spa": arr(sp["spa"]), "abvdem": arr(sp["abvdem"]), "spe": arr(sp["spe"]),
         "path": arr(sp["path"] + [path2]), "peth": arr(sp["peth"] + [peth2]), "dranu": arr([0.0] * 8),
         "vxf": FArray(np.linspace(-0.3, 0.7, tot))}
    for k in ("vnormf", "vtangf", "runiform", "vnormc", "vtangc", "psicos", "vnorms", "vtangs1", "vtangs2"):
        g[k] = arr([0.0] * tot)
    types = {k: "integer" for k in ("nspec", "is", "ns", "m", "iconf", "icon", "nprfrac1", "nprfrac2")}
    types.update({k: "real" for k in ("mainprop", "pi", "psi1", "psi2")})
    st = Stream(seed)
    it = Interpreter(u, g, st.externals(), types)
    nee = 0
    for s in range(ns):
        g["is"] = s + 1
        g["ns"] = nee + 1
        it.call("assign_velocity", [])
        nee += sp["npr"][s]
    for k in ("vnormf", "vtangf", "runiform", "vnormc", "vtangc", "psicos", "vnorms", "vtangs1", "vtangs2"):
        out[f"emit{variant}_{k}"] = g[k].data.copy()
    out[f"emit{variant}_case"] = np.array([seed, st.k, path2, peth2, 0.7], dtype=np.float64)
    out["emit_vxf"] = g["vxf"].data.copy()
    out["emit_species"] = np.array([[sp[k][s] for k in ("npr", "nphi", "spa", "abvdem", "spe", "peth", "path")]
                                    for s in range(ns)], dtype=np.float64)


def make(ref: Path) -> dict:
    out = {"stream_seed": np.array([4357.0]), "stream": O.ranu0_stream(4357, STREAM_PIN)}
    units = lemses_units(ref)
    run_builders(units, out)
    run_inflow(ref, units, out)
    run_emission(ref, units, out, 0, 700)
    run_emission(ref, units, out, 1, 701)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("EMSES_REFERENCE", str(HERE.parents[2] / "reference")),
                    help="the reference source tree ($EMSES_REFERENCE, else a `reference` directory beside "
                         "this repository)")
    args = ap.parse_args()
    out = make(Path(args.reference))
    np.savez_compressed(HERE / "tables.npz", **out)
    print({k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
