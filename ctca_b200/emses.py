"""Host-side mirror of the reference's particle-path subroutines over the C ABI.

The methods keep the reference's names and argument meaning:

    Emses.grdcrt(ps)                 subroutine grdcrt(ps)          src/field/grdcrt.F90:125
    Emses.psolve2(ps, ustep)         subroutine psolve2(ps, ustep)  src/pcl2field/psolve2.F90:4
    Emses.psolve1(ps, ustep, func)   subroutine psolve1(...)        src/pcl2field/psolve1.F90:4
    Emses.positn(ps, ustep)          subroutine positn(ps, ustep)   src/pcl/positn.F90:3
    Emses.charge(ps, func)           subroutine charge(ps, func)    src/pcl2field/charge.F90:4
    Emses.spsort(ps)                 subroutine spsort(ps)          src/etc/spsort.F90:4

Every call goes through libemsesg.so (CUDA kernels for sm_100a); there is no
CPU fallback, and the module refuses to load without the built library.
Errors from the library raise EmsesError with the library's message, as the
reference's `icon` / `errstop` paths report them.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

ISPEC = 10
INPC = 15

OK = 0
ERR_ARG = 1
ERR_UNSUPPORTED = 2
ERR_CUDA = 3
ERR_OVERFLOW = 4
ERR_NOMEM = 5
ERR_TIMEOUT = 6
ERR_DEVICE = 7
ERR_STATE = 8

PCL_ALIVE = 0
PCL_INJECTED = 1
PCL_TO_BE_ACCUMULATED = -1
PCL_TO_BE_ACCUMULATED_AS_ANTIPCL = -2

# Slots per row of the FP32 form's thread-major tile regions (EMSESG_FX_ROW_SLOTS).
FX_ROW_SLOTS = 736

FIELDS = {"eb": 0, "wrk": 1, "aj": 2, "ajdg": 3, "rho": 4, "rhodg": 5, "rhobk": 6, "rhobksp": 7, "phi": 8}

# oh_particle (lib/ohhelp/ohhelp-1.1.1/oh_type.F90:15-28): 64 bytes.
PARTICLE_DTYPE = np.dtype([("x", "<f8"), ("y", "<f8"), ("z", "<f8"), ("vx", "<f8"), ("vy", "<f8"),
                           ("vz", "<f8"), ("pid", "<i4"), ("preside", "<i4"), ("nid", "<i4"), ("spec", "<i4")])
assert PARTICLE_DTYPE.itemsize == 64


class Body(ctypes.Structure):
    _fields_ = [("geotype", ctypes.c_int32), ("ncond", ctypes.c_int32), ("cyl_align", ctypes.c_int32),
                ("reserved_", ctypes.c_int32),
                ("xlpc", ctypes.c_double), ("xupc", ctypes.c_double), ("ylpc", ctypes.c_double),
                ("yupc", ctypes.c_double), ("zlpc", ctypes.c_double), ("zupc", ctypes.c_double),
                ("cyl_axis", ctypes.c_double * 2), ("cyl_edge", ctypes.c_double * 2), ("radius", ctypes.c_double),
                ("sph_center", ctypes.c_double * 3), ("sqdscaled", ctypes.c_double)]


class Config(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
                ("nspec", ctypes.c_int32), ("nfbnd", ctypes.c_int32 * 3),
                ("npbnd", (ctypes.c_int32 * 3) * ISPEC), ("npc", ctypes.c_int32), ("line_mode", ctypes.c_int32),
                ("rng_mode", ctypes.c_int32), ("sort_tile", ctypes.c_int32 * 3), ("flags", ctypes.c_int32),
                ("rng_seed", ctypes.c_uint64), ("q", ctypes.c_double * ISPEC), ("qm", ctypes.c_double * ISPEC),
                ("rm", ctypes.c_double * ISPEC), ("e0", ctypes.c_double * 3), ("b0", ctypes.c_double * 3),
                ("body", Body * INPC), ("capacity", ctypes.c_int64 * ISPEC)]


class Counter(ctypes.Structure):
    """The Fortran sequence type `counter` (src/main/paramt.F90:76-83)."""
    _fields_ = [("globalp", (ctypes.c_int64 * ISPEC) * 2), ("influx", (ctypes.c_int32 * INPC) * ISPEC),
                ("outflux", (ctypes.c_int32 * INPC) * ISPEC),
                ("infhist", ((ctypes.c_int32 * (INPC + 1)) * INPC) * ISPEC),
                ("nesc", ctypes.c_int32 * ((ISPEC + 1) // 2 * 2)), ("chgacm", (ctypes.c_double * 2) * INPC)]

    def as_dict(self) -> dict:
        return {
            "influx": np.ctypeslib.as_array(self.influx).copy(),
            "infhist": np.ctypeslib.as_array(self.infhist).copy(),
            "nesc": np.ctypeslib.as_array(self.nesc).copy(),
            "chgacm": np.ctypeslib.as_array(self.chgacm).copy(),
        }


class Plasma(ctypes.Structure):
    _fields_ = [("ppc", ctypes.c_int32 * ISPEC), ("vth", ctypes.c_double * ISPEC),
                ("vdrift", (ctypes.c_double * 3) * ISPEC), ("seed", ctypes.c_uint64)]


# Declarations of include/emses_gpu.h, in order.
_P = ctypes.c_void_p
_I = ctypes.c_int
_SIGS = {
    "emsesg_select_device": (_I, [_I]),
    "emsesg_create": (_I, [ctypes.POINTER(Config), ctypes.POINTER(_P)]),
    "emsesg_destroy": (_I, [_P]),
    "emsesg_last_error": (_I, [_P, ctypes.c_char_p, ctypes.c_size_t]),
    "emsesg_stream": (_P, [_P]),
    "emsesg_synchronize": (_I, [_P]),
    "emsesg_field_size": (_I, [_P, _I, ctypes.POINTER(ctypes.c_int64)]),
    "emsesg_upload_particles": (_I, [_P, _I, _P, ctypes.POINTER(ctypes.c_int64)]),
    "emsesg_download_particles": (_I, [_P, _I, _P, ctypes.POINTER(ctypes.c_int64)]),
    "emsesg_upload_field": (_I, [_P, _I, _P]),
    "emsesg_download_field": (_I, [_P, _I, _P]),
    "emsesg_zero_field": (_I, [_P, _I]),
    "emsesg_set_counters": (_I, [_P, ctypes.POINTER(Counter)]),
    "emsesg_get_counters": (_I, [_P, ctypes.POINTER(Counter)]),
    "emsesg_set_randoms": (_I, [_P, _P, ctypes.c_int64]),
    "emsesg_grdcrt": (_I, [_P, _I]),
    "emsesg_psolve2": (_I, [_P, _I, _I, ctypes.POINTER(Counter)]),
    "emsesg_positn": (_I, [_P, _I, _I, ctypes.POINTER(Counter)]),
    "emsesg_psolve1": (_I, [_P, _I, _I, _I, ctypes.POINTER(Counter)]),
    "emsesg_charge": (_I, [_P, _I, _I]),
    "emsesg_reduce_rho": (_I, [_P, _I]),
    "emsesg_reduce_aj": (_I, [_P]),
    "emsesg_reduce_ajdg": (_I, [_P]),
    "emsesg_spsort": (_I, [_P, _I]),
    "emsesg_compact": (_I, [_P, _I, ctypes.POINTER(ctypes.c_int64)]),
    "emsesg_rhoupd": (_I, [_P, _I]),
    "emsesg_compact_noalloc": (_I, [_P, ctypes.c_int64, _P, _P, _P]),
    "emsesg_bfield": (_I, [_P, _I]),
    "emsesg_efield": (_I, [_P, _I, ctypes.c_double, ctypes.c_double]),
    "emsesg_exchange_eb": (_I, [_P]),
    "emsesg_fx_em_step": (_I, [_P, _I, _I, ctypes.c_double]),
    "emsesg_esfield": (_I, [_P, _P, _P, _I, _P]),
    "emsesg_fx_step_es": (_I, [_P, _I, _I]),
    "emsesg_energy": (_I, [_P, ctypes.POINTER(ctypes.c_double)]),
    "emsesg_fx_load": (_I, [_P]),
    "emsesg_fx_store": (_I, [_P]),
    "emsesg_fx_step": (_I, [_P, _I, _I]),
    "emsesg_fx_sort": (_I, [_P]),
    "emsesg_fx_run": (_I, [_P, _I, _I, _I, _I]),
    "emsesg_fx_chunk_rows": (_I, [_P, _I]),
    "emsesg_fx_step_download": (_I, [_P, _I, _I, _P, _P]),
    "emsesg_upload_field_async": (_I, [_P, _I, _P]),
    "emsesg_fx_slab": (_I, [_P, _I, ctypes.c_int64]),
    "emsesg_fx_slab_begin": (_I, [_P, _I, _P]),
    "emsesg_fx_slab_outbox": (_I, [_P, _I, _I, ctypes.POINTER(ctypes.c_void_p)]),
    "emsesg_fx_slab_planes": (_I, [_P, _I, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_int64),
                                   ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_int64)]),
    "emsesg_fx_slab_arrive": (_I, [_P, _I, ctypes.c_void_p, ctypes.c_int64]),
    "emsesg_fx_slab_border": (_I, [_P]),
    "emsesg_fx_slab_end": (_I, [_P, _I]),
    "emsesg_batch_create": (_I, [_P, _I, _I, _I, _P, ctypes.POINTER(_P)]),
    "emsesg_batch_launch": (_I, [_P, _I]),
    "emsesg_batch_stream": (_P, [_P]),
    "emsesg_batch_kernels": (_I, [_P, ctypes.POINTER(ctypes.c_int64)]),
    "emsesg_batch_destroy": (_I, [_P]),
    "emsesg_fx_counts": (_I, [_P, ctypes.POINTER(ctypes.c_int64)]),
    "emsesg_fx_download_accum": (_I, [_P, _P]),
    "emsesg_fx_inject": (_I, [_P, _I, _P, ctypes.c_int64]),
    "emsesg_fx_surface": (_I, [_P, _P, ctypes.POINTER(ctypes.c_int64)]),
    "emsesg_fx_background": (_I, [_P, _I]),
    "emsesg_fx_energy": (_I, [_P, ctypes.POINTER(ctypes.c_double)]),
    "emsesg_fx_continuity": (_I, [_P, ctypes.POINTER(ctypes.c_double)]),
    "emsesg_fx_emit": (_I, [_P, _I, _I, ctypes.c_double, _P, _P, ctypes.c_int64, _P, _P, _I, ctypes.c_uint64,
                            ctypes.c_uint64, ctypes.c_uint64]),
    "emsesg_fx_inflow_z": (_I, [_P, _I, _I, ctypes.c_int64, _P, _P, _P, _I, ctypes.c_double, ctypes.c_uint64,
                                ctypes.c_uint64, ctypes.c_uint64]),
    "emsesg_fx_inflow": (_I, [_P, _I, _I, _I, ctypes.c_int64, _P, _P, _P, _I, ctypes.c_double, ctypes.c_uint64,
                              ctypes.c_uint64, ctypes.c_uint64]),
    "emsesg_fx_emit_plane": (_I, [_P, _I, _I, ctypes.c_double, _P, _P, ctypes.c_int64, _P, _P, _I, ctypes.c_double,
                                  _I, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64]),
    "emsesg_fx_inflow_current": (_I, [_P, _I, _I, _I, ctypes.c_int64, _P, _P, _P, _I, ctypes.c_double, _I,
                                      ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64]),
    "emsesg_fx_emit_cylinder": (_I, [_P, _I, _I, _I, ctypes.c_double, _P, _I, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_double, ctypes.c_double, ctypes.c_int64, _P, _P, _P, _P, _P, _P, _I, _I,
                                     ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64]),
    "emsesg_fx_adjoint": (_I, [_P, _I, _I, _I, _I, _P, _P, ctypes.POINTER(ctypes.c_double), _P, _P, _P, _P]),
    "emsesg_load_plasma": (_I, [_P, ctypes.POINTER(Plasma)]),
    "emsesg_fx_load_plasma": (_I, [_P, ctypes.POINTER(Plasma)]),
    "emsesg_set_profiling": (_I, [_P, _I]),
    "emsesg_profile_report": (_I, [_P, ctypes.c_char_p, ctypes.c_size_t]),
    "emsesg_profile_reset": (_I, [_P]),
}

LIB_PATH = Path(__file__).resolve().parent / "libemsesg.so"
_lib = None


def library_path() -> Path:
    return Path(os.environ.get("EMSESG_LIB", LIB_PATH))


def load_library() -> ctypes.CDLL:
    """Loads libemsesg.so; raises ImportError when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not path.exists():
        raise ImportError(f"{path} is missing: build it with `python -m ctca_b200.build`")
    lib = ctypes.CDLL(str(path))
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def declared_symbols() -> list[str]:
    return list(_SIGS)


def select_device(device: int):
    """CUDA device for the contexts this thread creates next (local rank)."""
    rc = load_library().emsesg_select_device(int(device))
    if rc != OK:
        raise EmsesError(rc, f"cannot select CUDA device {device}")


class EmsesError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def field_extents(cfg: Config, name: str) -> tuple[int, int, int, int, int]:
    """(ncomp, lo, ext_x, ext_y, ext_z) of a field array (Fortran layout)."""
    nx, ny, nz, ns = cfg.nx, cfg.ny, cfg.nz, cfg.nspec
    return {
        "eb": (6, -1, nx + 3, ny + 3, nz + 3),
        "wrk": (9, -4, nx + 9, ny + 9, nz + 9),
        "aj": (3, -4, nx + 9, ny + 9, nz + 9),
        "ajdg": (3 * ns, -4, nx + 9, ny + 9, nz + 9),
        "rho": (1, -1, nx + 3, ny + 3, nz + 3),
        "rhodg": (2 * ns + 1, -1, nx + 3, ny + 3, nz + 3),
        "rhobk": (1, -1, nx + 3, ny + 3, nz + 3),
        "rhobksp": (1, -1, nx + 3, ny + 3, nz + 3),
        "phi": (1, -1, nx + 3, ny + 3, nz + 3),
    }[name]


def field_shape(cfg: Config, name: str) -> tuple[int, ...]:
    """numpy (C-order) shape of a field: (z, y, x, comp), plus a leading
    species axis for rhobksp.  Index [k-lo, j-lo, i-lo, c] is Fortran
    field(c+1, i, j, k)."""
    nc, lo, ex, ey, ez = field_extents(cfg, name)
    shp = (ez, ey, ex, nc)
    return (cfg.nspec,) + shp if name == "rhobksp" else shp


class Emses:
    """One device context (one rank, ps = 1) of the EMSES particle path."""

    def __init__(self, cfg: Config):
        self.lib = load_library()
        self.cfg = cfg
        h = ctypes.c_void_p()
        rc = self.lib.emsesg_create(ctypes.byref(cfg), ctypes.byref(h))
        if rc != OK:
            raise EmsesError(rc, "emsesg_create failed (bad configuration or no CUDA device)")
        self.h = h

    # -- plumbing
    def close(self):
        if getattr(self, "h", None):
            self.lib.emsesg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int):
        if rc != OK:
            buf = ctypes.create_string_buffer(512)
            self.lib.emsesg_last_error(self.h, buf, 512)
            raise EmsesError(rc, buf.value.decode(errors="replace"))

    @property
    def stream(self) -> int:
        return self.lib.emsesg_stream(self.h) or 0

    def synchronize(self):
        self._check(self.lib.emsesg_synchronize(self.h))

    # -- explicit sync points
    def upload_particles(self, pbuf: np.ndarray, totalp, ps: int = 1):
        pbuf = np.ascontiguousarray(pbuf, dtype=PARTICLE_DTYPE)
        tp = (ctypes.c_int64 * ISPEC)(*[int(t) for t in totalp])
        self._check(self.lib.emsesg_upload_particles(self.h, ps, pbuf.ctypes.data, tp))

    def download_particles(self, ps: int = 1):
        tp = (ctypes.c_int64 * ISPEC)()
        self._check(self.lib.emsesg_download_particles(self.h, ps, None, tp))
        total = sum(tp[: self.cfg.nspec])
        out = np.zeros(total, dtype=PARTICLE_DTYPE)
        self._check(self.lib.emsesg_download_particles(self.h, ps, out.ctypes.data, tp))
        return out, np.array(tp[: self.cfg.nspec], dtype=np.int64)

    def field_size(self, name: str) -> int:
        n = ctypes.c_int64()
        self._check(self.lib.emsesg_field_size(self.h, FIELDS[name], ctypes.byref(n)))
        return n.value

    def upload_field(self, name: str, arr: np.ndarray):
        a = np.ascontiguousarray(arr, dtype=np.float64).reshape(-1)
        if a.size != self.field_size(name):
            raise ValueError(f"{name}: expected {self.field_size(name)} doubles, got {a.size}")
        self._check(self.lib.emsesg_upload_field(self.h, FIELDS[name], a.ctypes.data))

    def download_field(self, name: str) -> np.ndarray:
        out = np.zeros(field_shape(self.cfg, name), dtype=np.float64)
        self._check(self.lib.emsesg_download_field(self.h, FIELDS[name], out.ctypes.data))
        return out

    def zero_field(self, name: str):
        self._check(self.lib.emsesg_zero_field(self.h, FIELDS[name]))

    def set_counters(self, gc: Counter):
        self._check(self.lib.emsesg_set_counters(self.h, ctypes.byref(gc)))

    def get_counters(self) -> Counter:
        gc = Counter()
        self._check(self.lib.emsesg_get_counters(self.h, ctypes.byref(gc)))
        return gc

    def set_randoms(self, u: np.ndarray):
        u = np.ascontiguousarray(u, dtype=np.float64)
        self._check(self.lib.emsesg_set_randoms(self.h, u.ctypes.data if u.size else None, u.size))

    # -- the reference subroutines
    def grdcrt(self, ps: int = 1):
        self._check(self.lib.emsesg_grdcrt(self.h, ps))

    def psolve2(self, ps: int, ustep: int, gcount: Counter | None = None):
        self._check(self.lib.emsesg_psolve2(self.h, ps, ustep, ctypes.byref(gcount) if gcount else None))

    def positn(self, ps: int, ustep: int, gcount: Counter | None = None):
        self._check(self.lib.emsesg_positn(self.h, ps, ustep, ctypes.byref(gcount) if gcount else None))

    def psolve1(self, ps: int, ustep: int, func: int, gcount: Counter | None = None):
        self._check(self.lib.emsesg_psolve1(self.h, ps, ustep, func, ctypes.byref(gcount) if gcount else None))

    def charge(self, ps: int, func: int):
        self._check(self.lib.emsesg_charge(self.h, ps, func))

    def reduce_rho(self, name: str = "rho"):
        self._check(self.lib.emsesg_reduce_rho(self.h, FIELDS[name]))

    def reduce_aj(self):
        self._check(self.lib.emsesg_reduce_aj(self.h))

    def reduce_ajdg(self):
        self._check(self.lib.emsesg_reduce_ajdg(self.h))

    def spsort(self, ps: int = 1):
        self._check(self.lib.emsesg_spsort(self.h, ps))

    def compact(self, ps: int = 1) -> np.ndarray:
        tp = (ctypes.c_int64 * ISPEC)()
        self._check(self.lib.emsesg_compact(self.h, ps, tp))
        return np.array(tp[: self.cfg.nspec], dtype=np.int64)

    def rhoupd(self, ps: int = 1):
        self._check(self.lib.emsesg_rhoupd(self.h, ps))

    def bfield(self, ps: int = 1):
        self._check(self.lib.emsesg_bfield(self.h, ps))

    def efield(self, ps: int, tcs: float, dlt: float = 2.0):
        self._check(self.lib.emsesg_efield(self.h, ps, tcs, dlt))

    def exchange_eb(self):
        self._check(self.lib.emsesg_exchange_eb(self.h))

    def fx_step_es(self, ustep: int, do_sort: bool):
        """The electrostatic step (psolve2 + charge): push and rho, no J."""
        self._check(self.lib.emsesg_fx_step_es(self.h, ustep, 1 if do_sort else 0))

    def fx_em_step(self, ustep: int, do_sort: bool, tcs: float):
        """bfield, fx_step, bfield, efield, exchange_eb (the main loop's order)."""
        self._check(self.lib.emsesg_fx_em_step(self.h, ustep, 1 if do_sort else 0, tcs))

    def esfield(self, mltstp: int = 1, check: bool = True, mtd_vbnd=(0, 0, 0), bc=None):
        """The electrostatic field from rho (esfld1(0) + poisson + esfld2):
        phi and EX..EZ of eb on the device.  mtd_vbnd per axis (0 periodic,
        1 phi = 0 on the faces, 2 Neumann); bc[axis][side] the Neumann values
        (boundary_conditions * rene).  With check, returns poichk's residual."""
        r = ctypes.c_double()
        t = (ctypes.c_int * 3)(*[int(x) for x in mtd_vbnd])
        b = None
        if bc is not None:
            b = (ctypes.c_double * 6)(*[float(bc[d][s]) for d in range(3) for s in range(2)])
        self._check(self.lib.emsesg_esfield(self.h, t, b, int(mltstp), ctypes.byref(r) if check else None))
        return r.value if check else None

    def energy(self) -> np.ndarray:
        e = (ctypes.c_double * (3 * ISPEC))()
        self._check(self.lib.emsesg_energy(self.h, e))
        return np.array(e[: 3 * self.cfg.nspec]).reshape(self.cfg.nspec, 3)

    # -- FP32 / fixed-point form
    def fx_load(self):
        self._check(self.lib.emsesg_fx_load(self.h))

    def fx_store(self):
        self._check(self.lib.emsesg_fx_store(self.h))

    def fx_step(self, ustep: int = 2, do_sort: bool = False):
        self._check(self.lib.emsesg_fx_step(self.h, ustep, 1 if do_sort else 0))

    def fx_step_download(self, ustep: int, do_sort: bool, rho: np.ndarray, aj: np.ndarray):
        """A step with rho and aj copied into the given host arrays (float64,
        contiguous, the fields' sizes) while the sort runs."""
        assert rho.dtype == np.float64 and aj.dtype == np.float64
        assert rho.size == self.field_size("rho") and aj.size == self.field_size("aj")
        self._check(self.lib.emsesg_fx_step_download(self.h, ustep, 1 if do_sort else 0, rho.ctypes.data,
                                                     aj.ctypes.data))

    def upload_eb_async(self, eb: np.ndarray):
        """The eb of the next step, copied beside the current step's sort
        (keep the array unchanged until the next step has started)."""
        assert eb.dtype == np.float64 and eb.size == self.field_size("eb") and eb.flags["C_CONTIGUOUS"]
        self._check(self.lib.emsesg_upload_field_async(self.h, FIELDS["eb"], eb.ctypes.data))

    def fx_chunk_rows(self, rows: int):
        """Rows of a tile region per push CTA (default 256)."""
        self._check(self.lib.emsesg_fx_chunk_rows(self.h, rows))

    # -- slab mode (a z slab of a decomposed grid; ctca_b200/slabs.py)
    def fx_slab(self, on: bool, outbox_cap: int = 0):
        self._check(self.lib.emsesg_fx_slab(self.h, 1 if on else 0, outbox_cap))

    def fx_slab_begin(self, ustep: int = 2) -> np.ndarray:
        """The push of a slab step; returns the particles leaving, [spec, dir]."""
        out = np.zeros(2 * ISPEC, dtype=np.int64)
        self._check(self.lib.emsesg_fx_slab_begin(self.h, ustep, out.ctypes.data))
        return out[:2 * self.cfg.nspec].reshape(self.cfg.nspec, 2)

    def fx_slab_outbox(self, spec: int, direction: int) -> int:
        """Device address of the outbox records of species spec, direction 0
        (through z = 0) or 1 (through z = nz)."""
        ptr = ctypes.c_void_p(0)
        self._check(self.lib.emsesg_fx_slab_outbox(self.h, spec, direction, ctypes.byref(ptr)))
        return ptr.value or 0

    def fx_slab_planes(self, which: int) -> tuple[int, int, int, int]:
        """(rho address, rho int64 count, J address, J int64 count) of the z
        border planes: which 0 sent down, 1 sent up, 2 received from below,
        3 received from above."""
        pr, pj = ctypes.c_void_p(0), ctypes.c_void_p(0)
        nr, nj = ctypes.c_int64(0), ctypes.c_int64(0)
        self._check(self.lib.emsesg_fx_slab_planes(self.h, which, ctypes.byref(pr), ctypes.byref(nr),
                                                   ctypes.byref(pj), ctypes.byref(nj)))
        return pr.value or 0, nr.value, pj.value or 0, nj.value

    def fx_slab_arrive(self, spec: int, dev_ptr: int, n: int):
        """Particles of species spec arriving from a neighbouring slab
        (n records at a device address)."""
        self._check(self.lib.emsesg_fx_slab_arrive(self.h, spec, ctypes.c_void_p(dev_ptr), n))

    def fx_slab_border(self):
        """The x / y border exchange of a slab step (after the arrivals,
        before the z border planes go to the neighbours)."""
        self._check(self.lib.emsesg_fx_slab_border(self.h))

    def fx_slab_end(self, do_sort: bool = False):
        self._check(self.lib.emsesg_fx_slab_end(self.h, 1 if do_sort else 0))

    def fx_run(self, ustep: int, nsteps: int, sort_every: int, use_graph: bool = True):
        """nsteps steps, re-sort every sort_every, replayed from a CUDA graph."""
        self._check(self.lib.emsesg_fx_run(self.h, ustep, nsteps, sort_every, 1 if use_graph else 0))

    def fx_sort(self):
        self._check(self.lib.emsesg_fx_sort(self.h))

    def fx_counts(self) -> np.ndarray:
        tp = (ctypes.c_int64 * ISPEC)()
        self._check(self.lib.emsesg_fx_counts(self.h, tp))
        return np.array(tp[: self.cfg.nspec], dtype=np.int64)

    def fx_download_accum(self) -> tuple[np.ndarray, np.ndarray]:
        nr = int(np.prod(field_shape(self.cfg, "rho")))
        nj = int(np.prod(field_shape(self.cfg, "aj")))
        out = np.zeros(nr + nj, dtype=np.int64)
        self._check(self.lib.emsesg_fx_download_accum(self.h, out.ctypes.data))
        return out[:nr].reshape(field_shape(self.cfg, "rho")), out[nr:].reshape(field_shape(self.cfg, "aj"))

    # -- synthetic loader and profile
    def fx_inject(self, spec: int, records: np.ndarray):
        """Injected particles of species `spec` (1-based): oh2_inject_particle."""
        rec = np.ascontiguousarray(records, dtype=PARTICLE_DTYPE)
        self._check(self.lib.emsesg_fx_inject(self.h, spec, rec.ctypes.data if rec.size else None, rec.size))

    def fx_inject_raw(self, spec: int, ptr: int, n: int):
        """fx_inject from a host address of n records (pinned memory: the
        upload is asynchronous; keep the records until the stream is past it)."""
        self._check(self.lib.emsesg_fx_inject(self.h, spec, ptr if n else None, n))

    def fx_emit(self, spec: int, nemd: int, grd: float, bounds1, bounds2, n: int, vnormf, vtangf,
                seed: int, stream: int, index0: int = 0):
        """n emitted pairs from a body face drawn on the device
        (emit_rectangle with hash_uniforms(seed, stream, index0, n, 6))."""
        b1 = (ctypes.c_double * 2)(*bounds1)
        b2 = (ctypes.c_double * 2)(*bounds2)
        vn = np.ascontiguousarray(vnormf, dtype=np.float64)
        vt = np.ascontiguousarray(vtangf, dtype=np.float64)
        assert vn.size == vt.size
        self._check(self.lib.emsesg_fx_emit(self.h, spec, nemd, grd, b1, b2, n, vn.ctypes.data, vt.ctypes.data,
                                            vn.size, seed, stream, index0))

    def fx_inflow_z(self, spec: int, front: bool, n: int, vz_table, vx_table, vy_table, injctisw: float,
                    seed: int, stream: int, index0: int = 0):
        """n inflow particles through a z face drawn on the device
        (inflow_z with hash_uniforms(seed, stream, index0, n, 5))."""
        t = [np.ascontiguousarray(x, dtype=np.float64) for x in (vz_table, vx_table, vy_table)]
        assert t[0].size == t[1].size == t[2].size
        self._check(self.lib.emsesg_fx_inflow_z(self.h, spec, 1 if front else 0, n, t[0].ctypes.data,
                                                t[1].ctypes.data, t[2].ctypes.data, t[0].size, injctisw, seed,
                                                stream, index0))

    def fx_emit_plane(self, spec: int, nemd: int, grd: float, b1, b2, n: int, vnorm, vtang, injctisw: float,
                      pid: int, seed: int, stream: int, index0: int = 0):
        """n particles emitted from a rectangular plane, drawn on the device
        (inject.emit_plane with hash_uniforms(seed, stream, index0, n, 6))."""
        vn = np.ascontiguousarray(vnorm, dtype=np.float64)
        vt = np.ascontiguousarray(vtang, dtype=np.float64)
        assert vn.size == vt.size
        cb1 = (ctypes.c_double * 2)(*b1)
        cb2 = (ctypes.c_double * 2)(*b2)
        self._check(self.lib.emsesg_fx_emit_plane(self.h, spec, nemd, grd, cb1, cb2, n, vn.ctypes.data,
                                                  vt.ctypes.data, vn.size, injctisw, pid, seed, stream, index0))

    def fx_emit_cylinder(self, spec: int, nemd: int, align: int, radius: float, axis, omni: int, grd: float,
                         hl: float, hu: float, psi: float, n: int, tabs: dict, anti: bool, seed: int, stream: int,
                         index0: int = 0):
        """n particles emitted from a face of a cylindrical body, drawn on the
        device (inject.emit_cylinder with hash_uniforms(seed, stream, index0,
        n, 6) flattened); tabs: vnormf, vtangf, runiform, vnormc, vtangc,
        psicos."""
        t = [np.ascontiguousarray(tabs[k], dtype=np.float64)
             for k in ("vnormf", "vtangf", "runiform", "vnormc", "vtangc", "psicos")]
        assert all(x.size == t[0].size for x in t)
        ax = (ctypes.c_double * 2)(*axis)
        self._check(self.lib.emsesg_fx_emit_cylinder(self.h, spec, nemd, align, radius, ax, omni, grd, hl, hu, psi, n,
                                                     *[x.ctypes.data for x in t], t[0].size, 1 if anti else 0, seed,
                                                     stream, index0))

    def fx_inflow(self, spec: int, axis: int, front: bool, n: int, vn_table, va_table, vb_table, injctisw: float,
                  seed: int, stream: int, index0: int = 0):
        """n inflow particles through a face of `axis` (0 x, 1 y, 2 z) drawn
        on the device (inject.inflow with hash_uniforms(seed, stream, index0,
        n, 5)); va / vb: the tangential tables of the other axes in order."""
        t = [np.ascontiguousarray(x, dtype=np.float64) for x in (vn_table, va_table, vb_table)]
        assert t[0].size == t[1].size == t[2].size
        self._check(self.lib.emsesg_fx_inflow(self.h, spec, axis, 1 if front else 0, n, t[0].ctypes.data,
                                              t[1].ctypes.data, t[2].ctypes.data, t[0].size, injctisw, seed,
                                              stream, index0))

    def fx_inflow_current(self, spec: int, axis: int, front: bool, n: int, vn_table, va_table, vb_table,
                          injctisw: float, ustep: int, seed: int, stream: int, index0: int = 0):
        """fx_inflow that also deposits psuper1's injection current into the
        J of the next step (inject.inflow_current times the charge)."""
        t = [np.ascontiguousarray(x, dtype=np.float64) for x in (vn_table, va_table, vb_table)]
        assert t[0].size == t[1].size == t[2].size
        self._check(self.lib.emsesg_fx_inflow_current(self.h, spec, axis, 1 if front else 0, n, t[0].ctypes.data,
                                                      t[1].ctypes.data, t[2].ctypes.data, t[0].size, injctisw,
                                                      ustep, seed, stream, index0))

    def fx_surface(self) -> np.ndarray:
        """Absorbed minus emitted particles per surface cell, [nspec, nsurf]."""
        n = ctypes.c_int64(0)
        self._check(self.lib.emsesg_fx_surface(self.h, None, ctypes.byref(n)))
        out = np.zeros((self.cfg.nspec, max(n.value, 0)), dtype=np.int64)
        if n.value:
            self._check(self.lib.emsesg_fx_surface(self.h, out.ctypes.data, ctypes.byref(n)))
        return out

    def fx_background(self, replace: bool = False):
        """add_background_charge of the FP32 form: rhobk from the surface
        counts, added into rho (or replacing it)."""
        self._check(self.lib.emsesg_fx_background(self.h, 1 if replace else 0))

    def fx_energy(self) -> np.ndarray:
        """Kinetic energy of the FP32 state in FP64, [nspec, 3] (energy)."""
        e = (ctypes.c_double * (3 * ISPEC))()
        self._check(self.lib.emsesg_fx_energy(self.h, e))
        return np.array(e[: 3 * self.cfg.nspec]).reshape(self.cfg.nspec, 3)

    def fx_continuity(self) -> tuple[float, float]:
        """(max |rho_new - rho_old + 2 div J|, max |rho_new|) of the last step."""
        r = (ctypes.c_double * 2)()
        self._check(self.lib.emsesg_fx_continuity(self.h, r))
        return float(r[0]), float(r[1])

    def fx_adjoint(self, K: int, ustep: int, ckpt: int, sort_every: int, probe_lo, probe_hi, nparticles: int,
                   gv_out: np.ndarray | None = None):
        """Loss sum_steps sum_probe aj_x^2 over K steps and its gradients:
        returns (loss, gE, gB, g0, gv) with node gradients [n^3, 3] and gv
        [nparticles, 3] in emsesg_fx_store order.  gv_out: a float64
        [nparticles, 3] buffer for gv (e.g. pinned host memory, so that its
        copy from the device runs at full speed)."""
        nn = self.cfg.nx * self.cfg.ny * self.cfg.nz
        gE = np.zeros((nn, 3))
        gB = np.zeros((nn, 3))
        g0 = np.zeros(6)
        if gv_out is not None:
            if gv_out.dtype != np.float64 or gv_out.shape != (nparticles, 3) or not gv_out.flags.c_contiguous:
                raise ValueError("gv_out must be a C-contiguous float64 array of shape (nparticles, 3)")
            gv = gv_out
        else:
            gv = np.zeros((nparticles, 3))
        loss = ctypes.c_double(0.0)
        lo = (ctypes.c_int32 * 3)(*probe_lo)
        hi = (ctypes.c_int32 * 3)(*probe_hi)
        self._check(self.lib.emsesg_fx_adjoint(self.h, K, ustep, ckpt, sort_every, lo, hi, ctypes.byref(loss),
                                               gE.ctypes.data, gB.ctypes.data, g0.ctypes.data, gv.ctypes.data))
        return loss.value, gE, gB, g0, gv

    def load_plasma(self, pl: Plasma):
        self._check(self.lib.emsesg_load_plasma(self.h, ctypes.byref(pl)))

    def fx_load_plasma(self, pl: Plasma):
        """The plasma of load_plasma straight into the FP32 form (no FP64 records)."""
        self._check(self.lib.emsesg_fx_load_plasma(self.h, ctypes.byref(pl)))

    def set_profiling(self, on: bool):
        self._check(self.lib.emsesg_set_profiling(self.h, 1 if on else 0))

    def profile(self) -> dict[str, tuple[float, int]]:
        buf = ctypes.create_string_buffer(1 << 16)
        self._check(self.lib.emsesg_profile_report(self.h, buf, 1 << 16))
        out = {}
        for line in buf.value.decode().splitlines():
            name, ms, n = line.split()
            out[name] = (float(ms), int(n))
        return out

    def profile_reset(self):
        self._check(self.lib.emsesg_profile_reset(self.h))


class Batch:
    """One CUDA graph holding `block` steps of each of several runs
    (emsesg_batch_create); `launch(nrep)` replays it nrep times."""

    def __init__(self, runs: list, ustep: int, block: int, sort_every: list):
        self.lib = load_library()
        self.runs = list(runs)
        n = len(self.runs)
        hs = (ctypes.c_void_p * n)(*[r.h.value for r in self.runs])
        se = (ctypes.c_int * n)(*[int(x) for x in sort_every])
        h = ctypes.c_void_p()
        rc = self.lib.emsesg_batch_create(ctypes.cast(hs, ctypes.c_void_p), n, ustep, block,
                                          ctypes.cast(se, ctypes.c_void_p), ctypes.byref(h))
        if rc != OK:
            self._raise(rc)
        self.h = h
        self.block = block

    def _raise(self, rc: int):
        for r in self.runs:
            buf = ctypes.create_string_buffer(512)
            self.lib.emsesg_last_error(r.h, buf, 512)
            if buf.value:
                raise EmsesError(rc, buf.value.decode(errors="replace"))
        raise EmsesError(rc, "emsesg_batch call failed")

    @property
    def stream(self) -> int:
        return self.lib.emsesg_batch_stream(self.h) or 0

    @property
    def kernels(self) -> int:
        """Kernel launches in one replay of the graph."""
        n = ctypes.c_int64(0)
        rc = self.lib.emsesg_batch_kernels(self.h, ctypes.byref(n))
        if rc != OK:
            self._raise(rc)
        return n.value

    def launch(self, nrep: int):
        rc = self.lib.emsesg_batch_launch(self.h, int(nrep))
        if rc != OK:
            self._raise(rc)

    def close(self):
        if getattr(self, "h", None):
            self.lib.emsesg_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
