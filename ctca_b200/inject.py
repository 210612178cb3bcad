"""Host-side particle supervisors of the injection rows: face emission from a
box body (psuper3.F90:142-239) and open-boundary inflow along z
(psuper2.F90:236-292).  They produce oh_particle records for
Emses.fx_inject (emsesg_fx_inject); the reference's supervisors also run on
the host and hand each new particle to oh2_inject_particle.

Velocity tables.  The reference fills vnormf / vtangf / vzf / vzb / vxr / vyr
at initialisation (src/main/inipin.F90:476-660, 996-1097) and the
supervisors draw table entries with addr = nprs + npr*U; the tables are
built by the reference's own table code, restated in ctca_b200/tables.py
(vflux / RANN0 / rexch on the reference's Mersenne Twister stream).

Random numbers come from a numpy Generator (the reference uses MT19937
through RANU0), or, with `uniforms=`, from a given array; the number and
order of draws per particle follow the reference: 6 per emitted particle
(u(4) unused), 5 per inflow particle.  `hash_uniforms` gives the draws of
the device supervisors (emsesg_fx_emit / emsesg_fx_inflow_z), so the two
produce the same records.
"""
from __future__ import annotations


import numpy as np

from .emses import PARTICLE_DTYPE

PCL_INJECTED = 1
PCL_ANTI = -2


_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def _mix64(z: np.ndarray) -> np.ndarray:
    """SplitMix64 finaliser (Steele, Lea, Flood 2014) on uint64 arrays."""
    z = z + np.uint64(0x9E3779B97F4A7C15)
    z = (z ^ (z >> np.uint64(30))) * _M1
    z = (z ^ (z >> np.uint64(27))) * _M2
    return z ^ (z >> np.uint64(31))


def hash_uniforms(seed: int, stream: int, index0: int, n: int, per: int) -> np.ndarray:
    """[n, per] U[0,1) numbers with 53 random bits: element (k, c) is the
    counter hash of (seed, stream, (index0 + k) * per + c), the draws of the
    device supervisors."""
    with np.errstate(over="ignore"):
        a = _mix64(np.uint64(seed) ^ _mix64(np.array([stream], dtype=np.uint64) + np.uint64(0x632BE59BD9B4E019)))
        idx = (np.uint64(index0) + np.arange(n, dtype=np.uint64)[:, None]) * np.uint64(per) + \
            np.arange(per, dtype=np.uint64)[None, :]
        b = _mix64(a ^ (idx * np.uint64(0xD1B54A32D192ED03)))
    return (b >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def emission_count(istep: int, lstep: int, fluxf: float, injct: int, ustep: int) -> int:
    """nemit of psuper3.F90:64-66."""
    return (int((istep + lstep) * fluxf) - int((istep + lstep - injct) * fluxf)) * ustep


# nemd -> (normal axis, sign); tangential axes follow psuper3.F90:152-185:
# +-1: (vx | vy, vz), +-2: (vy | vz, vx), +-3: (vz | vx, vy)
_ORDER = {1: (0, 1, 2), 2: (1, 2, 0), 3: (2, 0, 1)}


# The twin's offset from the face: psuper3.F90:196-206 adds the literal 1e-5,
# a default (single precision) real in the reference's build, to a double.
TWIN_OFFSET = float(np.float32(1e-5))


def emit_rectangle(nemd: int, grd: float, bounds1: tuple, bounds2: tuple, n: int, vnormf: np.ndarray,
                   vtangf: np.ndarray, rng: np.random.Generator | None, spec: int,
                   uniforms: np.ndarray | None = None) -> np.ndarray:
    """n emitted particles from a rectangular face (emit_from_rectangle,
    psuper3.F90:142-208): each gives an anti-particle (preside -2) on the
    face and its twin 1e-5 off the face along the normal (preside +1).
    bounds1 / bounds2 are the face extents along the first / second
    tangential axis of nemd.  Returns 2n records, anti-particle first."""
    axis = _ORDER[abs(nemd)]
    ud = 1.0 if nemd > 0 else -1.0
    npr = vnormf.size
    u = rng.random((n, 6)) if uniforms is None else uniforms
    out = np.zeros(2 * n, dtype=PARTICLE_DTYPE)  # pid = nid = 0
    coords = [("x", "vx"), ("y", "vy"), ("z", "vz")]
    a0 = (npr * u[:, 0]).astype(np.int64)
    a1 = (npr * u[:, 1]).astype(np.int64)
    a2 = (npr * u[:, 2]).astype(np.int64)
    vn = ud * vnormf[a0]
    vt1 = vtangf[a1]
    vt2 = vtangf[a2]
    rn = np.full(n, grd)
    rt1 = bounds1[0] + (bounds1[1] - bounds1[0]) * u[:, 4]
    rt2 = bounds2[0] + (bounds2[1] - bounds2[0]) * u[:, 5]
    # whole-field writes of the interleaved pairs (anti-particle, twin)
    for val_r, val_v, ax in ((rn, vn, axis[0]), (rt1, vt1, axis[1]), (rt2, vt2, axis[2])):
        c, v = coords[ax]
        r2 = np.repeat(val_r, 2)
        if ax == axis[0]:
            r2[1::2] += ud * TWIN_OFFSET
        out[c] = r2
        out[v] = np.repeat(val_v, 2)
    out["preside"] = np.tile(np.array([PCL_ANTI, PCL_INJECTED], dtype=np.int32), n)
    out["spec"] = spec
    return out


def _flat_uniforms(n: int, rng, uniforms) -> np.ndarray:
    """The 6n numbers of one emission call (RANU0(dranu, n*6)), flat."""
    if uniforms is not None:
        return np.asarray(uniforms, dtype=np.float64).ravel()
    return rng.random(6 * n)


# The side surface of a cylinder of axis `align`: the emission routine's
# (normal, first tangential, second tangential) axes and which of the
# cylinder's two axis coordinates give the first two (psuper3.F90:301-346).
_CYL_SIDE = {1: ((2, 1, 0), (1, 0)), 2: ((2, 0, 1), (0, 1)), 3: ((0, 1, 2), (0, 1))}


def emit_cylinder(nemd: int, align: int, radius: float, axis: tuple, omni: int, grd: float, hl: float, hu: float,
                  psi: float, n: int, tabs: dict, rng: np.random.Generator | None, spec: int,
                  uniforms: np.ndarray | None = None, anti: bool = True) -> np.ndarray:
    """n particles emitted from a cylindrical body (emit_from_cylinder,
    psuper3.F90:241-371) from 6n uniforms u (the flat RANU0 array of the
    call).  A face nemd along the cylinder's axis (|nemd| = align) is an end
    cap (emit_from_circular_surf, :373-410): normal speed ud *
    vnormf[int(npr u0)], tangential vtangf[int(npr u1)], vtangf[int(npr u2)];
    the point at grd on the normal axis and radius * runiform[int(npr u3)]
    from the axis (axis[0], axis[1]) at the angle 2 pi u4.  Any other face is
    the side surface, by omni and radius (:412-528): radius >= 1
    (emit_from_cylindrical_surf1) turns vnormc / vtangc by psicos + psi and
    puts the point on the circle at that angle; radius < 1 (surf2, five
    uniforms a particle) turns them by psi and puts the point where the
    velocity's direction meets the circle; omni = 1 (surf3) turns them by an
    azimuth 2 pi u2; the coordinate along the axis is hl + (hu - hl) u5 (u4
    for surf2).  Each particle gives a record with preside 1 and, with
    `anti` (ncond <= 0), its anti-particle (preside -2) at the same place.
    tabs: vnormf, vtangf, runiform, vnormc, vtangc, psicos (one species,
    tables.emission_tables).  The trigonometry is the C library's."""
    import math
    u = _flat_uniforms(n, rng, uniforms)
    vnormf, vtangf, runiform = tabs["vnormf"], tabs["vtangf"], tabs["runiform"]
    vnormc, vtangc, psicos = tabs["vnormc"], tabs["vtangc"], tabs["psicos"]
    npr = vnormf.size
    pi2 = math.pi * 2.0
    cap = abs(nemd) == align
    ud = 1.0 if nemd > 0 else -1.0
    per = 5 if (not cap and omni == 0 and radius < 1.0) else 6
    out = np.zeros(2 * n if anti else n, dtype=PARTICLE_DTYPE)
    coords = (("x", "vx"), ("y", "vy"), ("z", "vz"))
    for m in range(n):
        ir = per * m
        ad = [int(npr * float(u[ir + c])) for c in range(4)]
        if cap:
            perm = _ORDER[abs(nemd)]
            vn, vt1, vt2 = ud * vnormf[ad[0]], vtangf[ad[1]], vtangf[ad[2]]
            radial = radius * runiform[ad[3]]
            angular = pi2 * float(u[ir + 4])
            rn, rt1, rt2 = grd, axis[0] + radial * math.cos(angular), axis[1] + radial * math.sin(angular)
        else:
            perm, (k1, k2) = _CYL_SIDE[align]
            a1, a2 = axis[k1], axis[k2]
            if omni == 0 and radius >= 1.0:
                ang = psicos[ad[2]] + psi
                vn = vnormc[ad[0]] * math.cos(ang) - vtangc[ad[1]] * math.sin(ang)
                vt1 = vnormc[ad[0]] * math.sin(ang) + vtangc[ad[1]] * math.cos(ang)
                rn, rt1 = a1 + radius * math.cos(ang), a2 + radius * math.sin(ang)
                vt2 = vtangf[ad[3]]
                rt2 = hl + (hu - hl) * float(u[ir + 5])
            elif omni == 0:
                vn = vnormc[ad[0]] * math.cos(psi) - vtangc[ad[1]] * math.sin(psi)
                vt1 = vnormc[ad[0]] * math.sin(psi) + vtangc[ad[1]] * math.cos(psi)
                vt2 = vtangf[ad[2]]
                v2normi = radius / math.sqrt(vn * vn + vt1 * vt1)
                rn, rt1 = a1 + vn * v2normi, a2 + vt1 * v2normi
                rt2 = hl + (hu - hl) * float(u[ir + 4])
            else:
                eaz = pi2 * float(u[ir + 2])
                vn = vnormc[ad[0]] * math.cos(eaz) - vtangc[ad[1]] * math.sin(eaz)
                vt1 = vnormc[ad[0]] * math.sin(eaz) + vtangc[ad[1]] * math.cos(eaz)
                vt2 = vtangf[ad[3]]
                rn, rt1 = a1 + radius * math.cos(eaz), a2 + radius * math.sin(eaz)
                rt2 = hl + (hu - hl) * float(u[ir + 5])
        k = 2 * m if anti else m
        for val_r, val_v, ax in ((rn, vn, perm[0]), (rt1, vt1, perm[1]), (rt2, vt2, perm[2])):
            c, v = coords[ax]
            out[c][k] = val_r
            out[v][k] = val_v
            if anti:
                out[c][k + 1] = val_r
                out[v][k + 1] = val_v
        out["preside"][k] = PCL_INJECTED
        if anti:
            out["preside"][k + 1] = PCL_ANTI
    out["spec"] = spec
    return out


def emit_plane(nemd: int, grd: float, bounds1: tuple, bounds2: tuple, n: int, vnormf: np.ndarray,
               vtangf: np.ndarray, injctisw: float, rng: np.random.Generator | None, spec: int, pid: int = 0,
               uniforms: np.ndarray | None = None) -> np.ndarray:
    """n particles emitted from a rectangular plane of a body
    (emit_from_rectangular_surf, psuper2.F90:330-360, 554-576): per particle
    six uniforms; normal speed ud * vnormf[int(npr*u0)], tangential speeds
    vtangf[int(npr*u1)], vtangf[int(npr*u2)]; the normal coordinate
    grd + vnorm * injctisw * u3 and the tangential ones uniform on the plane
    (u4, u5) plus vtang * injctisw * u3: the particle has flown for the
    fraction u3 of the injection interval.  One record per particle (no
    anti-particle), pid = the body, preside 0."""
    axis = _ORDER[abs(nemd)]
    ud = 1.0 if nemd > 0 else -1.0
    npr = vnormf.size
    u = rng.random((n, 6)) if uniforms is None else uniforms
    out = np.zeros(n, dtype=PARTICLE_DTYPE)
    coords = [("x", "vx"), ("y", "vy"), ("z", "vz")]
    a0 = (npr * u[:, 0]).astype(np.int64)
    a1 = (npr * u[:, 1]).astype(np.int64)
    a2 = (npr * u[:, 2]).astype(np.int64)
    vn = ud * vnormf[a0]
    vt1 = vtangf[a1]
    vt2 = vtangf[a2]
    rn = grd + vn * injctisw * u[:, 3]
    rt1 = bounds1[0] + (bounds1[1] - bounds1[0]) * u[:, 4] + vt1 * injctisw * u[:, 3]
    rt2 = bounds2[0] + (bounds2[1] - bounds2[0]) * u[:, 5] + vt2 * injctisw * u[:, 3]
    for val_r, val_v, ax in ((rn, vn, axis[0]), (rt1, vt1, axis[1]), (rt2, vt2, axis[2])):
        c, v = coords[ax]
        out[c] = val_r
        out[v] = val_v
    out["spec"] = spec
    out["pid"] = pid
    return out


def inflow_count(istep: int, lstep: int, arr: float, injct: int, ustep: int) -> int:
    """narrzf / narrzb of psuper2.F90:238-239, 266-267."""
    return (int((istep + lstep) * arr) - int((istep + lstep - injct) * arr)) * ustep


def inflow(axis: int, front: bool, n: int, nx: int, ny: int, nz: int, vn_table: np.ndarray, va_table: np.ndarray,
           vb_table: np.ndarray, injctisw: float, rng: np.random.Generator | None, spec: int,
           zssurf: float = -1.0e30, uniforms: np.ndarray | None = None) -> np.ndarray:
    """Particles entering through the lower (front) or upper face of `axis`
    (0: x, 1: y, 2: z), psuper2.F90:114-292 (x faces :114-173, y :175-233, z
    :236-292).  Per particle five uniforms: u0 picks the normal speed
    vn_table[int(npr*u0)], u1 the tangential ones va_table / vb_table
    [int(npr*u1)] (the two other axes in increasing order), u2 / u3 / u4 give
    x / y / z: uniform on the face along the tangential axes, and along the
    normal the distance vn * injctisw * u covered within the last injctisw
    steps, from 0 or from the upper face.  preside 0.  Like the reference,
    a particle with z <= zssurf is dropped whatever the face."""
    npr = vn_table.size
    u = rng.random((n, 5)) if uniforms is None else uniforms
    a1 = (npr * u[:, 0]).astype(np.int64)
    a2 = (npr * u[:, 1]).astype(np.int64)
    out = np.zeros(n, dtype=PARTICLE_DTYPE)
    ext = (nx, ny, nz)
    names = ("x", "y", "z")
    vn = vn_table[a1]
    tang = [d for d in range(3) if d != axis]
    for d in range(3):
        if d == axis:
            out[names[d]] = (vn * injctisw * u[:, 2 + d]) if front else (ext[d] + vn * injctisw * u[:, 2 + d])
        else:
            out[names[d]] = 0.0 + ext[d] * u[:, 2 + d]
    out["v" + names[axis]] = vn
    out["v" + names[tang[0]]] = va_table[a2]
    out["v" + names[tang[1]]] = vb_table[a2]
    out["spec"] = spec
    keep = out["z"] > zssurf
    return out[keep]


# (normal, first, second) axes of the zigzag weights of J along each axis:
# Jx is spread over (j, k), Jy over (i, k), Jz over (i, j)
_ZZ_SPREAD = ((1, 2), (0, 2), (0, 1))


def _zigzag_add(wrk: np.ndarray, b: list, a: list, rustep: float) -> None:
    """One particle's zigzag current from b to a (psuper1.F90:859-988,
    current_deposition) added into wrk[k + 4, j + 4, i + 4, comp] in the
    reference's order (segment b -> relay point, then relay point -> a; per
    segment the weights 1..4, each for x, y, z)."""
    import math
    ib = [math.floor(v) for v in b]
    ia = [math.floor(v) for v in a]
    r = [(b[d] + a[d]) * 0.5 if ib[d] == ia[d] else max(float(ib[d]), float(ia[d])) for d in range(3)]
    for cell, dd, vv in ((ib, [(r[d] + b[d]) * 0.5 - float(ib[d]) for d in range(3)],
                          [(r[d] - b[d]) * rustep for d in range(3)]),
                         (ia, [(a[d] + r[d]) * 0.5 - float(ia[d]) for d in range(3)],
                          [(a[d] - r[d]) * rustep for d in range(3)])):
        w = []
        for comp in range(3):
            e1, e2 = _ZZ_SPREAD[comp]
            w4 = dd[e1] * dd[e2]
            w2 = dd[e1] - w4
            w3 = dd[e2] - w4
            w1 = 1.0 - dd[e1] - w3
            w.append((w1, w2, w3, w4))
        for q in range(4):
            for comp in range(3):
                e1, e2 = _ZZ_SPREAD[comp]
                n = list(cell)
                if q & 1:
                    n[e1] += 1
                if q & 2:
                    n[e2] += 1
                wrk[n[2] + 4, n[1] + 4, n[0] + 4, comp] += vv[comp] * w[comp][q]


def inflow_current(axis: int, front: bool, rec: np.ndarray, ustep: int, ext: tuple,
                   wrk: np.ndarray | None = None) -> np.ndarray:
    """The injection current of psuper1 (psuper1.F90:120-323 with
    current_deposition, :859-988) for records `rec` injected through the
    lower (front) or upper face of `axis`, in order: the zigzag current of
    the path from b to the injection point a, b outside the face (-1 below
    the lower face, n + 0.99999999 above the upper one, along the normal;
    a - v * ustep along the other axes), without the charge factor (the
    reference's wrk(TJX:TJZ), added to aj times q).  Returns (or adds into)
    wrk, numpy (nz + 9, ny + 9, nx + 9, 3) over the nodes -4..n+4 of each
    axis."""
    nx, ny, nz = ext
    if wrk is None:
        wrk = np.zeros((nz + 9, ny + 9, nx + 9, 3))
    rustep = 1.0 / ustep
    names = ("x", "y", "z")
    for p in rec:
        a = [float(p[c]) for c in names]
        b = [a[d] - float(p["v" + names[d]]) * ustep for d in range(3)]
        b[axis] = -1.0 if front else ext[axis] + 0.99999999
        _zigzag_add(wrk, b, a, rustep)
    return wrk


def inflow_z(front: bool, n: int, nx: int, ny: int, nz: int, vz_table: np.ndarray, vx_table: np.ndarray,
             vy_table: np.ndarray, injctisw: float, rng: np.random.Generator | None, spec: int,
             zssurf: float = -1.0e30, uniforms: np.ndarray | None = None) -> np.ndarray:
    """Particles entering through the z = 0 face (front) or z = nz face
    (back), psuper2.F90:236-292: inflow(2, ...)."""
    return inflow(2, front, n, nx, ny, nz, vz_table, vx_table, vy_table, injctisw, rng, spec, zssurf, uniforms)
