"""TEST INFRASTRUCTURE ONLY: Python binding of the CPU oracle (liboracle.so).

The oracle is the FP64 restatement of the reference's particle path
(emses_oracle.cpp).  Only tests/, __graft_entry__.smoke() and the CPU
baseline of bench.py use it, and only as the checker or the timed CPU
reference; the product (ctca_b200) never imports it.

Also binds oracle/_ref/libemses_ref.so, the reference's own C sources for
this path (MT19937 of lib/mtarm, particle_sort_ of lib/psort) when built.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

from ctca_b200.emses import ISPEC, PARTICLE_DTYPE, Config, Counter, Plasma, field_shape

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF_LIB = HERE / "_ref" / "libemses_ref.so"
FIELD_IDS = {"eb": 0, "wrk": 1, "aj": 2, "ajdg": 3, "rho": 4, "rhodg": 5, "rhobk": 6, "rhobksp": 7}

_P = ctypes.c_void_p
_lib = None


def reference_dir() -> Path:
    """The reference's source tree: $EMSES_REFERENCE, else a `reference`
    directory beside this repository."""
    env = os.environ.get("EMSES_REFERENCE")
    return Path(env) if env else HERE.parent.parent / "reference"


def build(reference: str | None = None):
    """Builds liboracle.so (and _ref/ when the reference sources exist)."""
    args = ["make", "-C", str(HERE), "liboracle.so"]
    subprocess.run(args, check=True, capture_output=True)
    ref = Path(reference) if reference else reference_dir()
    if (ref / "lib" / "mtarm" / "mt19937arm.c").exists():
        subprocess.run(["make", "-C", str(HERE), "ref", f"REFERENCE={ref}"], check=True, capture_output=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB.exists():
        build()
    L = ctypes.CDLL(str(LIB))
    cfgp = ctypes.POINTER(Config)
    i64p = ctypes.POINTER(ctypes.c_int64)
    sigs = {
        "orc_field_size": (ctypes.c_int64, [cfgp, ctypes.c_int]),
        "orc_exchange_eb": (None, [cfgp, _P]),
        "orc_bfield": (None, [cfgp, _P]),
        "orc_efield": (None, [cfgp, _P, _P, ctypes.c_double, ctypes.c_double]),
        "orc_grdcrt": (None, [cfgp, _P, _P]),
        "orc_psolve2": (ctypes.c_int, [cfgp, ctypes.c_int, _P, _P, i64p, _P, ctypes.c_int64, i64p, ctypes.c_uint64,
                                       ctypes.POINTER(Counter)]),
        "orc_positn": (ctypes.c_int, [cfgp, ctypes.c_int, _P, i64p, _P, ctypes.c_int64, i64p, ctypes.c_uint64,
                                      ctypes.POINTER(Counter)]),
        "orc_psolve1": (ctypes.c_int, [cfgp, ctypes.c_int, ctypes.c_int, _P, _P, i64p, _P, ctypes.c_int64, i64p,
                                       ctypes.c_uint64, _P, _P, ctypes.POINTER(Counter), _P]),
        "orc_surface_layout": (ctypes.c_int64, [cfgp, _P]),
        "orc_surface_cell": (ctypes.c_int64, [cfgp, ctypes.c_int, _P, _P]),
        "orc_surface_point": (ctypes.c_int64, [cfgp, ctypes.c_int, _P]),
        "orc_background": (None, [cfgp, _P, _P, _P, ctypes.c_int]),
        "orc_charge": (None, [cfgp, ctypes.c_int, _P, i64p, _P, _P, _P, _P]),
        "orc_reduce_rho": (None, [cfgp, _P, ctypes.c_int]),
        "orc_reduce_aj": (None, [cfgp, _P]),
        "orc_reduce_ajdg": (None, [cfgp, _P]),
        "orc_rhoupd": (None, [cfgp, _P, _P]),
        "orc_energy": (None, [cfgp, _P, i64p, _P]),
        "orc_sort_key": (ctypes.c_int64, [cfgp, _P]),
        "orc_spsort": (None, [cfgp, _P, i64p]),
        "orc_compact": (None, [cfgp, _P, i64p]),
        "orc_hash_u01": (ctypes.c_double, [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64]),
        "orc_load_plasma": (None, [cfgp, ctypes.POINTER(Plasma), _P, i64p]),
        "orc_adjoint": (ctypes.c_double, [cfgp, ctypes.c_int, ctypes.c_int, _P, _P, _P, _P, ctypes.c_int64, _P, _P,
                                          _P, _P, _P, _P]),
        "orc_adjoint_ckpt": (ctypes.c_double, [cfgp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _P, _P, _P, _P,
                                               ctypes.c_int64, _P, _P, _P, _P, _P, _P]),
        "orc_zigzag_one": (None, [cfgp, ctypes.c_int, ctypes.c_double, _P, _P, _P]),
        "orc_blocks_create": (_P, [cfgp, _P, _P, i64p, ctypes.c_int, ctypes.c_int]),
        "orc_blocks_threads": (ctypes.c_int, [_P]),
        "orc_blocks_particles": (ctypes.c_int64, [_P]),
        "orc_blocks_step": (ctypes.c_double, [_P, ctypes.c_int, ctypes.c_int]),
        "orc_blocks_result": (None, [_P, _P, _P]),
        "orc_blocks_destroy": (None, [_P]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _tp(totalp) -> ctypes.Array:
    return (ctypes.c_int64 * ISPEC)(*[int(t) for t in totalp])


def zeros(cfg: Config, name: str) -> np.ndarray:
    return np.zeros(field_shape(cfg, name), dtype=np.float64)


class Oracle:
    """Holds the CPU state of one rank: pbuf, wrk, aj, ajdg, rho, ... ."""

    def __init__(self, cfg: Config, pbuf: np.ndarray, totalp, eb: np.ndarray):
        self.cfg = cfg
        self.L = lib()
        self.pbuf = np.ascontiguousarray(pbuf, dtype=PARTICLE_DTYPE).copy()
        self.totalp = np.array(totalp, dtype=np.int64)
        self.eb = np.ascontiguousarray(eb, dtype=np.float64).copy()
        self.f = {name: zeros(cfg, name) for name in FIELD_IDS if name != "eb"}
        self.gc = Counter()
        self.nsurf = int(self.L.orc_surface_layout(ctypes.byref(cfg), None))
        self.surf = np.zeros((cfg.nspec, max(self.nsurf, 1)), dtype=np.int64)
        self.ranu = np.zeros(0)
        self.ranu_pos = ctypes.c_int64(0)
        self.rng_stream = 0

    def _c(self):
        return ctypes.byref(self.cfg)

    def set_randoms(self, u):
        self.ranu = np.ascontiguousarray(u, dtype=np.float64)
        self.ranu_pos = ctypes.c_int64(0)

    def grdcrt(self):
        self.L.orc_grdcrt(self._c(), self.eb.ctypes.data, self.f["wrk"].ctypes.data)

    def psolve2(self, ustep: int):
        tp = _tp(self.totalp)
        rc = self.L.orc_psolve2(self._c(), ustep, self.f["wrk"].ctypes.data, self.pbuf.ctypes.data, tp,
                                self.ranu.ctypes.data if self.ranu.size else None, self.ranu.size,
                                ctypes.byref(self.ranu_pos), self.rng_stream, ctypes.byref(self.gc))
        self.rng_stream += 1
        if rc:
            raise RuntimeError("oracle psolve2: random numbers exhausted")

    def positn(self, ustep: int):
        tp = _tp(self.totalp)
        rc = self.L.orc_positn(self._c(), ustep, self.pbuf.ctypes.data, tp,
                               self.ranu.ctypes.data if self.ranu.size else None, self.ranu.size,
                               ctypes.byref(self.ranu_pos), self.rng_stream, ctypes.byref(self.gc))
        self.rng_stream += 1
        if rc:
            raise RuntimeError("oracle positn: random numbers exhausted")

    def psolve1(self, ustep: int, func: int = 0):
        tp = _tp(self.totalp)
        rc = self.L.orc_psolve1(self._c(), ustep, func, self.f["wrk"].ctypes.data, self.pbuf.ctypes.data, tp,
                                self.ranu.ctypes.data if self.ranu.size else None, self.ranu.size,
                                ctypes.byref(self.ranu_pos), self.rng_stream, self.f["aj"].ctypes.data,
                                self.f["ajdg"].ctypes.data, ctypes.byref(self.gc), self.surf.ctypes.data)
        self.rng_stream += 1
        if rc:
            raise RuntimeError("oracle psolve1: random numbers exhausted")

    def charge(self, func: int = 0):
        tp = _tp(self.totalp)
        self.L.orc_charge(self._c(), func, self.pbuf.ctypes.data, tp, self.f["rho"].ctypes.data,
                          self.f["rhodg"].ctypes.data, self.f["rhobk"].ctypes.data, self.f["rhobksp"].ctypes.data)

    def reduce_rho(self, name: str = "rho"):
        a = self.f[name]
        nc = a.shape[-1]
        if name == "rhobksp":
            for s in range(a.shape[0]):
                sub = np.ascontiguousarray(a[s])
                self.L.orc_reduce_rho(self._c(), sub.ctypes.data, nc)
                a[s] = sub
        else:
            self.L.orc_reduce_rho(self._c(), a.ctypes.data, nc)

    def bfield(self):
        self.L.orc_bfield(self._c(), self.eb.ctypes.data)

    def efield(self, tcs: float, dlt: float = 2.0):
        self.L.orc_efield(self._c(), self.eb.ctypes.data, self.f["aj"].ctypes.data, tcs, dlt)

    def exchange_eb(self):
        self.L.orc_exchange_eb(self._c(), self.eb.ctypes.data)

    def reduce_aj(self):
        self.L.orc_reduce_aj(self._c(), self.f["aj"].ctypes.data)

    def reduce_ajdg(self):
        self.L.orc_reduce_ajdg(self._c(), self.f["ajdg"].ctypes.data)

    def rhoupd(self):
        self.L.orc_rhoupd(self._c(), self.f["rho"].ctypes.data, self.f["aj"].ctypes.data)

    def background(self, surf=None, replace: bool = False):
        """rhobk from the surface counts (the oracle's own, or `surf`), added
        into rho (add_background_charge)."""
        s = np.ascontiguousarray(self.surf if surf is None else surf, dtype=np.int64)
        self.L.orc_background(self._c(), s.ctypes.data, self.f["rhobk"].ctypes.data, self.f["rho"].ctypes.data,
                              int(replace))

    def energy(self) -> np.ndarray:
        e = np.zeros(3 * ISPEC)
        self.L.orc_energy(self._c(), self.pbuf.ctypes.data, _tp(self.totalp), e.ctypes.data)
        return e[: 3 * self.cfg.nspec].reshape(self.cfg.nspec, 3)

    def spsort(self):
        self.L.orc_spsort(self._c(), self.pbuf.ctypes.data, _tp(self.totalp))

    def compact(self):
        tp = _tp(self.totalp)
        self.L.orc_compact(self._c(), self.pbuf.ctypes.data, tp)
        self.totalp = np.array(tp[: self.cfg.nspec], dtype=np.int64)
        self.pbuf = self.pbuf[: int(self.totalp.sum())].copy()

    def sort_keys(self) -> np.ndarray:
        return np.array([self.L.orc_sort_key(self._c(), self.pbuf[m:m + 1].ctypes.data)
                         for m in range(self.pbuf.size)], dtype=np.int64)


def exchange_eb(cfg: Config, eb: np.ndarray) -> np.ndarray:
    out = np.ascontiguousarray(eb, dtype=np.float64).copy()
    lib().orc_exchange_eb(ctypes.byref(cfg), out.ctypes.data)
    return out


def hash_u01(seed: int, stream: int, index: int) -> float:
    return lib().orc_hash_u01(seed, stream, index)


def load_plasma(cfg: Config, pl: Plasma):
    n = int(sum(pl.ppc[i] for i in range(cfg.nspec))) * cfg.nx * cfg.ny * cfg.nz
    pbuf = np.zeros(n, dtype=PARTICLE_DTYPE)
    tp = (ctypes.c_int64 * ISPEC)()
    lib().orc_load_plasma(ctypes.byref(cfg), ctypes.byref(pl), pbuf.ctypes.data, tp)
    return pbuf, np.array(tp[: cfg.nspec], dtype=np.int64)


class Blocks:
    """The timed CPU baseline (baseline.cpp): the reference's one rank per
    core, each owning a block of x rows of the grid with its own sub-grid
    arrays, running psolve1 + charge on its particles.  `wrk` is the global
    node field (grdcrt output)."""

    def __init__(self, cfg: Config, wrk: np.ndarray, pbuf: np.ndarray, totalp, threads: int, margin: int = 3):
        self.cfg = cfg
        self.L = lib()
        p = np.ascontiguousarray(pbuf, dtype=PARTICLE_DTYPE)
        w = np.ascontiguousarray(wrk, dtype=np.float64)
        self.h = self.L.orc_blocks_create(ctypes.byref(cfg), w.ctypes.data, p.ctypes.data, _tp(totalp), threads,
                                          margin)
        self.threads = int(self.L.orc_blocks_threads(self.h))
        self.particles = int(self.L.orc_blocks_particles(self.h))

    def step(self, ustep: int = 2, restore: bool = True) -> float:
        """One step of every block (from the initial particles when
        `restore`); returns the wall seconds of psolve1 + charge."""
        return float(self.L.orc_blocks_step(self.h, ustep, int(restore)))

    def result(self):
        """aj and rho of the last step, folded periodically (interior nodes)."""
        aj, rho = zeros(self.cfg, "aj"), zeros(self.cfg, "rho")
        self.L.orc_blocks_result(self.h, aj.ctypes.data, rho.ctypes.data)
        return aj, rho

    def close(self):
        if self.h:
            self.L.orc_blocks_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


# -- the reference's own C code (oracle/_ref) --------------------------------
_ref = None


def ref_lib():
    """libemses_ref.so built from the reference's lib/mtarm and lib/psort."""
    global _ref
    if _ref is None:
        if not REF_LIB.exists():
            return None
        L = ctypes.CDLL(str(REF_LIB))
        L.mt_init_.argtypes = [ctypes.POINTER(ctypes.c_int)]
        L.mt_init_.restype = ctypes.c_int
        L.mtrand_real8_.argtypes = []
        L.mtrand_real8_.restype = ctypes.c_double
        L.particle_sort_.argtypes = [_P, ctypes.POINTER(ctypes.c_int)]
        L.particle_sort_.restype = None
        _ref = L
    return _ref


def ranu0_stream(seed: int, n: int) -> np.ndarray:
    """n successive RANU0 draws of the reference (randinit0 + mtrand_real8,
    src/wrapper/wrapper.F90:20-87 over lib/mtarm/mt19937arm.c)."""
    L = ref_lib()
    if L is None:
        raise RuntimeError("oracle/_ref not built")
    s = ctypes.c_int(seed)
    L.mt_init_(ctypes.byref(s))
    return np.array([L.mtrand_real8_() for _ in range(n)])


def adjoint(cfg: Config, K: int, ustep: int, enode: np.ndarray, bnode: np.ndarray, e0b0, pbuf: np.ndarray,
            probe_lo, probe_hi, grad: bool = True, ckpt: int = 0):
    """FP64 loss sum_steps sum_probe Jx^2 of K periodic steps and its
    gradients (adjoint.cpp): returns (loss, gE, gB, g0, gv); node fields are
    [n^3][3] with x fastest and exclude e0 / b0.  ckpt: keep the state every
    ckpt steps and recompute in between (0: keep every state)."""
    p = np.ascontiguousarray(pbuf, dtype=PARTICLE_DTYPE).copy()
    en = np.ascontiguousarray(enode, dtype=np.float64)
    bn = np.ascontiguousarray(bnode, dtype=np.float64)
    e0 = np.ascontiguousarray(e0b0, dtype=np.float64)
    lo = (ctypes.c_int * 3)(*probe_lo)
    hi = (ctypes.c_int * 3)(*probe_hi)
    nn = cfg.nx * cfg.ny * cfg.nz
    gE = np.zeros((nn, 3)) if grad else None
    gB = np.zeros((nn, 3)) if grad else None
    g0 = np.zeros(6) if grad else None
    gv = np.zeros((p.size, 3)) if grad else None
    ptr = (lambda a: a.ctypes.data if a is not None else None)
    loss = lib().orc_adjoint_ckpt(ctypes.byref(cfg), K, ckpt or K, ustep, en.ctypes.data, bn.ctypes.data,
                                  e0.ctypes.data, p.ctypes.data, p.size, lo, hi, ptr(gE), ptr(gB), ptr(g0), ptr(gv))
    return loss, gE, gB, g0, gv
