"""The reference's velocity tables for injection and emission, restated.

At initialisation the reference fills tables of npr velocities per species
(src/main/inipin.F90:476-660 for the open outer boundaries,
inipin.F90:996-1097 `assign_velocity` for emission from bodies) from its
table builders in src/etc/lemses.F90:
  vflux   (lemses.F90:361-425)  npr speeds of the flux through a face of a
                                drifting Maxwellian, by stepping through the
                                flux distribution in equal-probability cells
                                from its maximum outwards, then shuffled
  vinit   (lemses.F90:428-498)  npr speeds of a Maxwellian (xlos = 0) or of
                                a loss-cone distribution v^xlos exp(-v^2/vt^2)
  ringds  (lemses.F90:314-358)  npr speeds of a ring distribution
  rexch   (lemses.F90:184-311)  the shuffle: 4 rounds of n/2 swaps of random
                                pairs, the same pairs in every array given
  arange / arymod (lemses.F90:9-83)
and the normal deviates of RANN0 (src/wrapper/wrapper.F90:307-375, the
Box-Muller form of drann0l).  The supervisors then draw entry
nprs + int(npr * u) of a table.

All random numbers come from one stream, the reference's RANU0: MT19937
seeded with init_genrand(iseed) (src/main/inital.F90:708, randinit0) and
read as 53-bit doubles (genrand_res53, lib/mtarm/mt19937arm.c: M. Matsumoto
and T. Nishimura's published generator).  `Ranu0` is that stream (numpy's
legacy MT19937 seeding is init_genrand, and its random_sample is
genrand_res53).  Every routine here draws from it in the reference's order,
so a table built from the same seed after the same earlier draws is the
reference's table bit for bit; the arithmetic is the reference's, one IEEE
double operation at a time (no fused multiply-adds), with the C library's
exp, erf, sqrt, log, cos, sin and tgamma as gfortran calls them.
"""
from __future__ import annotations

import ctypes
import ctypes.util
import math

import numpy as np

PI_LEMSES = 3.14159265358979        # the literal of vflux / vinit / ringds
SQ2_LEMSES = 1.41421356237309       # the literal of vinit / ringds
PEI2 = 6.28318530717958646          # 2 pi of RANN0

_libm = None


def _tgamma(x: float) -> float:
    """GAMMA as gfortran evaluates it: the C library's tgamma."""
    global _libm
    if _libm is None:
        _libm = ctypes.CDLL(ctypes.util.find_library("m"))
        _libm.tgamma.restype = ctypes.c_double
        _libm.tgamma.argtypes = [ctypes.c_double]
    return _libm.tgamma(float(x))


def _nint(x: float) -> int:
    """NINT: to the nearest integer, halves away from zero."""
    return int(math.floor(x + 0.5)) if x >= 0 else -int(math.floor(-x + 0.5))


class Ranu0:
    """The reference's uniform stream: MT19937 with init_genrand(seed),
    53-bit doubles in [0, 1)."""

    def __init__(self, seed: int):
        self._rs = np.random.RandomState(int(seed) & 0xFFFFFFFF)
        self.drawn = 0

    def draw(self, n: int) -> np.ndarray:
        """RANU0(dranu, n, icon): the next n numbers."""
        n = int(n)
        self.drawn += n
        return self._rs.random_sample(n) if n > 0 else np.zeros(0)


def rexch(n: int, arrays: list, rng: Ranu0) -> None:
    """rexch (lemses.F90:184-311), in place: 4 rounds; a round draws n
    numbers and swaps, for i = 1..n/2, the entries int(n u(2i-1)) + 1 and
    int(n u(2i)) + 1 (1-based) of every array given."""
    n = int(n)
    nexch = n // 2
    arrs = [a for a in arrays if a is not None]
    for _ in range(4):
        u = rng.draw(n)
        for i in range(nexch):
            n1 = int(n * float(u[2 * i])) + 1
            n2 = int(n * float(u[2 * i + 1])) + 1
            if n1 <= 0 or n2 <= 0 or n1 > n or n2 > n:
                continue
            for a in arrs:
                t = a[n1 - 1]
                a[n1 - 1] = a[n2 - 1]
                a[n2 - 1] = t


def vflux(na: int, v0: float, vt: float, isl: int, rng: Ranu0) -> tuple[np.ndarray, int]:
    """vflux (lemses.F90:361-425): na speeds of the flux of a Maxwellian of
    drift v0 and thermal speed vt through a face, towards +v (isl = 1) or -v
    (isl = -1); returns (table, icon), icon the first entry left unset (0:
    all set).  The steps start at the maximum vm of v f(v) and go down to 0
    (each entry the mid-point of a cell of probability ts/na), then up."""
    na = int(na)
    ar = np.zeros(na)
    pi = PI_LEMSES
    aa = math.sqrt(2.0 / pi) * vt * math.exp(-((v0 / vt) * (v0 / vt)) * 0.5)
    bb = math.erf(v0 / (vt * math.sqrt(2.0)))
    ts = 0.0
    if isl == 1:
        ts = (aa + v0 * (1.0 + bb)) * 0.5
    if isl == -1:
        ts = (-aa + v0 * (1.0 - bb)) * 0.5
    dd = v0 * v0 + 4.0 * (vt * vt)
    vm = 0.0
    if v0 >= 0.0:
        if isl == 1:
            vm = (v0 + math.sqrt(dd)) * 0.5
        if isl == -1:
            vm = -2.0 * (vt * vt) / (v0 + math.sqrt(dd))
    else:
        if isl == -1:
            vm = (v0 - math.sqrt(dd)) * 0.5
        if isl == 1:
            vm = 2.0 * (vt * vt) / (v0 - math.sqrt(dd))
    ds = abs(ts) / na
    v1 = vm
    v2 = vm
    i = 1
    cc = 1.0 / (math.sqrt(2.0 * pi) * vt)

    def fl(v):
        r = (v - v0) / vt
        return cc * v * math.exp(-(r * r) * 0.5)

    done = False
    while True:  # downwards from the maximum
        ee = fl(v1)
        if ee == 0.0:
            break
        dvd = ds / ee
        v1 = v1 - dvd
        if isl == 1 and v1 <= 0.0:
            break
        if isl == -1 and v1 >= 0.0:
            break
        ar[i - 1] = v1 + 0.5 * dvd
        i += 1
    while True:  # upwards
        ee = fl(v2)
        if ee == 0.0:
            done = True
            break
        dvd = ds / ee
        v2 = v2 + dvd
        ar[i - 1] = v2 - 0.5 * dvd
        i += 1
        if i > na:
            break
    # entries not reached stay zero
    if done:
        ar[i - 1:] = 0.0
    icon = i if i < na else 0
    rexch(na, [ar], rng)
    return ar, icon


def vinit(na: int, v0: float, vt: float, xlos: float, rng: Ranu0) -> tuple[np.ndarray, float, float]:
    """vinit (lemses.F90:428-498): na speeds; xlos = 0: the Maxwellian of
    drift v0, entries v0 +- sqrt(2) vt x_k at equal-probability steps of
    exp(-x^2); else the loss-cone distribution v^|xlos| exp(-v^2/vt^2) (vt
    from v0 when xlos > 0, v0 from vt when xlos < 0, both returned as the
    reference updates its arguments).  Returns (table, v0, vt)."""
    na = int(na)
    ar = np.zeros(na)
    ppii = PI_LEMSES
    sq2 = SQ2_LEMSES
    if xlos == 0.0:
        vd = sq2 * vt
        nph = na // 2
        ds = math.sqrt(ppii) / na
        n = 0
        x = 0.0
        for _ in range(nph):
            dx = ds / math.exp(-(x * x))
            x = x + dx
            dvp = vd * (x - 0.5 * dx)
            ar[n] = v0 + dvp
            ar[n + 1] = v0 - dvp
            n += 2
        rexch(na, [ar], rng)
        return ar, v0, vt
    axlos = abs(xlos)
    if xlos > 0.0:
        vt = v0 * sq2 / math.sqrt(axlos)
    else:
        v0 = vt * math.sqrt(axlos) / sq2
    dv = vt
    a = 1.0 / (dv * dv)
    xx = 0.5 * (axlos + 1.0)
    xxm = -xx
    ts = 0.5 * (a ** xxm) * _tgamma(xx)
    ds = ts / na
    sqvc = axlos * 0.5 / a
    v1 = math.sqrt(sqvc)
    v2 = v1
    j = 1
    while True:
        avm = -a * v1 * v1
        fv1 = (v1 ** axlos) * math.exp(avm)
        dvd = ds / fv1
        v1 = v1 - dvd
        if v1 <= 0.0:
            break
        ar[j - 1] = v1 + 0.5 * dvd
        j += 1
    while True:
        avm = -a * v2 * v2
        fv2 = (v2 ** axlos) * math.exp(avm)
        dvd = ds / fv2
        v2 = v2 + dvd
        ar[j - 1] = v2 - 0.5 * dvd
        j += 1
        if j > na:
            break
    rexch(na, [ar], rng)
    return ar, v0, vt


def ringds(na: int, vt: float, bbb: float, rng: Ranu0) -> np.ndarray:
    """ringds (lemses.F90:314-358): na speeds of the ring distribution
    v (exp(-v^2/vt^2) - exp(-v^2/(bbb vt^2))) / (1 - bbb), shuffled."""
    na = int(na)
    ar = np.zeros(na)
    ds = vt * vt / 2.0 / na
    a = 1.0 / (vt * vt)
    cc = 1.0 / (1.0 - bbb)
    v1 = vt
    v2 = v1
    j = 1
    while True:
        avm = -a * v1 * v1
        fv1 = cc * v1 * (math.exp(avm) - math.exp(avm / bbb))
        dvd = ds / fv1
        v1 = v1 - dvd
        if v1 <= 0.0:
            break
        ar[j - 1] = v1 + 0.5 * dvd
        j += 1
    while True:
        avm = -a * v2 * v2
        fv2 = cc * v2 * (math.exp(avm) - math.exp(avm / bbb))
        dvd = ds / fv2
        v2 = v2 + dvd
        ar[j - 1] = v2 - 0.5 * dvd
        j += 1
        if j > na:
            break
    rexch(na, [ar], rng)
    return ar


def rann0(am: float, sd: float, n: int, rng: Ranu0) -> np.ndarray:
    """RANN0 (drann0l, wrapper.F90:307-375): n normal deviates of mean am
    and deviation sd, Box-Muller on pairs of uniforms (cos, then sin); an
    odd last one from two more uniforms."""
    n = int(n)
    out = np.zeros(n)
    if n == 1:
        w = rng.draw(2)
        out[0] = am + sd * math.sqrt(-2.0 * math.log(w[0])) * math.cos(PEI2 * w[1])
        return out
    odd = n % 2
    nn = n - odd
    u = rng.draw(nn)
    for i in range(0, nn, 2):
        w1 = sd * math.sqrt(-2.0 * math.log(float(u[i])))
        w2 = PEI2 * float(u[i + 1])
        out[i] = am + w1 * math.cos(w2)
        out[i + 1] = am + w1 * math.sin(w2)
    if odd:
        w = rng.draw(2)
        out[n - 1] = am + sd * math.sqrt(-2.0 * math.log(w[0])) * math.cos(PEI2 * w[1])
    return out


def arange_(aa: np.ndarray, nam: int, id_: int, rng: Ranu0) -> None:
    """arange (lemses.F90:9-54) in place: nothing for id <= 1; else the
    sorted table dealt out into id interleaved groups placed at shuffled
    starts, each group shuffled."""
    if id_ <= 1:
        return
    id_ = min(id_, 1024)
    aa[:nam] = np.sort(aa[:nam], kind="stable")
    ip = nam // id_
    if ip * id_ < nam:
        return
    iia = np.array([ip * k + 1 for k in range(id_)], dtype=np.int64)
    rexch(id_, [iia], rng)
    bb = aa[:nam].copy()
    js = 1
    for k in range(id_):
        j = js
        i = int(iia[k])
        i0 = i
        for _ in range(ip):
            aa[i - 1] = bb[j - 1]
            i += 1
            j += id_
        sub = aa[i0 - 1:i0 - 1 + ip]
        rexch(ip, [sub], rng)
        js += 1


def arymod(aa: np.ndarray, in_: int, nam: int, is_: int, id_: int) -> None:
    """arymod (lemses.F90:57-83) in place: the first nam entries spread to
    positions is, is + id, is + 2 id, ... (1-based); the others keep their
    values."""
    if in_ < nam * id_:
        return
    bb = aa[:nam].copy()
    i = is_
    for j in range(nam):
        aa[i - 1] = bb[j]
        i += id_


def signed_flux(npq: int, vd: float, vt: float, isl: int, rng: Ranu0) -> tuple[np.ndarray, int]:
    """A table of the flux towards +v (isl 1) or -v (isl -1) for a signed
    drift vd: inipin.F90:501-580 (negative drift: the mirrored table)."""
    if vd >= 0.0:
        return vflux(npq, vd, vt, isl, rng)
    t, icon = vflux(npq, -vd, vt, -isl, rng)
    return -t, icon


def inflow_tables(npr: int, nphi: int, vdt: tuple, peth: float, path: float, rng: Ranu0) -> dict:
    """The tables of one species injected through open outer boundaries
    (inipin.F90:492-652): vxf, vxb, vyf, vyb, vzf, vzb (flux through the
    lower / upper face of each axis; drift vdt, thermal speed peth along x
    and y, path along z), vxr, vyr, vzr (Maxwellians), each of npr entries
    with the first npr / nphi set, in the reference's order of draws; and
    icon of each flux table."""
    npq = int(npr) // int(nphi)
    out, icons = {}, {}
    for ax, name, vt in ((0, "x", peth), (1, "y", peth), (2, "z", path)):
        for side, isl in (("f", 1), ("b", -1)):
            t, icon = signed_flux(npq, vdt[ax], vt, isl, rng)
            tab = np.zeros(int(npr))
            tab[:npq] = t
            out[f"v{name}{side}"] = tab
            icons[f"v{name}{side}"] = icon
    for side in ("f", "b"):
        for name in "xyz":
            arange_(out[f"v{name}{side}"], npq, 1, rng)
        for name in "xyz":
            arymod(out[f"v{name}{side}"], int(npr), npq, 1, int(nphi))
    for ax, name, vt in ((0, "x", peth), (1, "y", peth), (2, "z", path)):
        tab = np.zeros(int(npr))
        tab[:npq] = rann0(vdt[ax], vt, npq, rng)
        out[f"v{name}r"] = tab
    rexch(npr, [out["vxf"], out["vxb"], out["vyf"], out["vyb"], out["vzf"], out["vzb"]], rng)
    rexch(npr, [out["vxr"], out["vyr"], out["vzr"]], rng)
    out["icon"] = icons
    return out


def inflow_rates(vdt: tuple, peth: float, path: float, npin: float, box: tuple, face: tuple, dt: float,
                 inpf: bool = True, inpb: bool = True) -> dict:
    """arrxf .. arrzb (inipin.F90:660-716): particles a step entering
    through the lower (f) and upper (b) face of each axis, for npin
    particles in the box (slx, sly, slz), faces of the extents face =
    (xu - xl, yu - yl, zu - zl) and step dt; zero for a side whose
    injection is off (inpf / inpb)."""
    slx, sly, slz = box
    ex, ey, ez = face
    pdf = abs(npin) / (slx * sly * slz)
    pdb = pdf
    ext = ((ey, ez), (ez, ex), (ex, ey))
    out = {}
    for ax, name, vt in ((0, "x", peth), (1, "y", peth), (2, "z", path)):
        vd = vdt[ax]
        aa = math.sqrt(2.0 / math.pi) * vt * math.exp(-((vd / vt) * (vd / vt)) * 0.5)
        bb = math.erf(vd / (math.sqrt(2.0) * vt))
        f = (aa + vd * (1.0 + bb)) * 0.5
        b = (-aa + vd * (1.0 - bb)) * 0.5
        e1, e2 = ext[ax]
        out[f"arr{name}f"] = abs(f) * pdf * e1 * e2 * dt * 0.5 if inpf else 0.0
        out[f"arr{name}b"] = abs(b) * pdb * e1 * e2 * dt * 0.5 if inpb else 0.0
    return out


def emission_tables(npr: int, npq: int, vnorm_drift: float, path: float, peth: float, spe: float,
                    rng: Ranu0, vxf: np.ndarray | None = None, path2: float = 0.0, peth2: float = 0.0,
                    mainprop: float = 1.0, emit: bool = True) -> dict:
    """The emission tables of one species (assign_velocity,
    inipin.F90:996-1097): vnormf (flux of drift spa + abvdem = vnorm_drift
    and thermal speed path; a second population of path2 for the fraction
    1 - mainprop when path2 > 0), vtangf (RANN0 of mean spe, deviation peth;
    peth2 likewise), runiform (sqrt-distributed radii), vnormc / vtangc
    (vnormf turned by an angle of density cos psi), psicos, and vnorms /
    vtangs1 / vtangs2 from vxf (the outer-boundary flux table, zero when not
    given).  `emit` false: no flux table (inpf(is) = 0).  Returns the
    tables and icon (non-zero: the flux table was not filled and the
    reference cancels this species' emission)."""
    npr = int(npr)
    vnormf = np.zeros(npr)
    icon = 0
    if path2 > 0.0:
        n1 = _nint(npr * mainprop)
        n2 = npr - n1
        if emit:
            t, icon = vflux(n1, vnorm_drift, path, 1, rng)
            vnormf[:n1] = t
        if icon != 0:
            emit = False
        if n2 > 0:
            if emit:
                t, icon = vflux(n2, vnorm_drift, path2, 1, rng)
                vnormf[n1:n1 + n2] = t
            if icon != 0:
                emit = False
    else:
        if emit:
            t, icon = vflux(npq, vnorm_drift, path, 1, rng)
            vnormf[:npq] = t
    rexch(npr, [vnormf], rng)
    rexch(npr, [vnormf], rng)
    vtangf = np.zeros(npr)
    if peth2 > 0.0:
        n1 = _nint(npr * mainprop)
        n2 = npr - n1
        vtangf[:n1] = rann0(spe, peth, n1, rng)
        if n2 > 0:
            vtangf[n1:n1 + n2] = rann0(spe, peth2, n2, rng)
    else:
        vtangf[:npq] = rann0(spe, peth, npq, rng)
    pi = math.pi
    runiform = np.zeros(npr)
    m = 0
    while m < npr:
        d = rng.draw(2)
        if d[1] <= d[0]:
            runiform[m] = d[0]
            m += 1
    vnormc = np.zeros(npr)
    vtangc = np.zeros(npr)
    m = 0
    while m < npr:
        d = rng.draw(2)
        psi1 = pi * (d[0] - 0.5)
        if d[1] <= math.cos(psi1):
            vtangc[m] = vnormf[m] * math.sin(psi1)
            vnormc[m] = vnormf[m] * math.cos(psi1)
            m += 1
    psicos = np.zeros(npr)
    m = 0
    while m < npr:
        d = rng.draw(2)
        psi1 = pi * (d[0] - 0.5)
        if d[1] <= math.cos(psi1):
            psicos[m] = psi1
            m += 1
    vx = np.zeros(npr) if vxf is None else np.asarray(vxf, dtype=np.float64)
    vnorms = np.zeros(npr)
    vtangs1 = np.zeros(npr)
    vtangs2 = np.zeros(npr)
    m = 0
    while m < npr:
        d = rng.draw(3)
        psi1 = pi * (d[0] - 0.5)
        if d[1] <= math.cos(psi1) * math.sin(psi1) * 2.0:
            t1 = vx[m] * math.sin(psi1)
            vnorms[m] = vx[m] * math.cos(psi1)
            psi2 = 2.0 * pi * d[2]
            vtangs2[m] = t1 * math.sin(psi2)
            vtangs1[m] = t1 * math.cos(psi2)
            m += 1
    return {"vnormf": vnormf, "vtangf": vtangf, "runiform": runiform, "vnormc": vnormc, "vtangc": vtangc,
            "psicos": psicos, "vnorms": vnorms, "vtangs1": vtangs1, "vtangs2": vtangs2, "icon": icon,
            "emit": emit}
