"""The host injection supervisors (ctca_b200/inject.py) against golden
vectors made by executing the reference's own psuper2.F90 text
(tests/golden/make_golden_supervisors.py): the inflow counts and records of
all six outer faces (psuper2.F90:114-292, with the z-surface drop) and the
rectangular-plane emission of every face orientation (:333-362, 554-576),
bit for bit on the same uniforms.  The device supervisors are checked
against these host ones by tests/test_gpu_supervisors.py."""
from pathlib import Path

import numpy as np
import pytest

from ctca_b200 import inject

GOLDEN = Path(__file__).resolve().parent / "golden" / "supervisors.npz"
KIN = ("x", "y", "z", "vx", "vy", "vz")


@pytest.fixture(scope="module")
def gold():
    if not GOLDEN.exists():
        pytest.skip("supervisors.npz not generated")
    return dict(np.load(GOLDEN))


def test_inflow_counts_and_records(gold):
    nx, ny, nz = (int(v) for v in gold["ext"])
    ustep, injct = int(gold["ustep"]), int(gold["injct"])
    istep, lstep = int(gold["istep"]), int(gold["lstep"])
    t = {k[4:]: gold[k] for k in gold if k.startswith("tab_")}
    # face order of psuper2: x-bottom, x-top, y-bottom, y-top, z-bottom, z-top
    faces = [("arrxf", 0, True, t["vxf"], t["vyr"], t["vzr"]), ("arrxb", 0, False, t["vxb"], t["vyr"], t["vzr"]),
             ("arryf", 1, True, t["vyf"], t["vxr"], t["vzr"]), ("arryb", 1, False, t["vyb"], t["vxr"], t["vzr"]),
             ("arrzf", 2, True, t["vzf"], t["vxr"], t["vyr"]), ("arrzb", 2, False, t["vzb"], t["vxr"], t["vyr"])]
    u = gold["uniforms"]
    pos = 0
    recs = []
    for key, axis, front, vn, va, vb in faces:
        n = inject.inflow_count(istep, lstep, float(gold["arr_" + key]), injct, ustep)
        assert n == int(gold["count_" + key]), key
        uu = u[pos:pos + 5 * n].reshape(n, 5)
        pos += 5 * n
        recs.append(inject.inflow(axis, front, n, nx, ny, nz, vn, va, vb, float(injct * ustep), None, spec=1,
                                  zssurf=float(gold["zssurf"]), uniforms=uu))
    assert pos == u.size
    got = np.concatenate(recs)
    want = gold["inflow_records"]
    assert got.size == want.size and got.size > 0
    assert want.size < sum(int(gold["count_" + f[0]]) for f in faces)  # the surface drop happened
    for f in KIN:
        assert np.array_equal(got[f], want[f]), f
    assert np.array_equal(got["preside"], want["preside"])
    assert np.array_equal(got["spec"], want["spec"])


def test_plane_emission_records(gold):
    n = int(gold["emit_n"])
    xl, xu, yl, yu, zl, zu = gold["emit_bounds"]
    tang = {1: ((yl, yu), (zl, zu)), 2: ((zl, zu), (xl, xu)), 3: ((xl, xu), (yl, yu))}
    injctisw = float(int(gold["injct"]) * int(gold["ustep"]))
    u = gold["emit_uniforms"]
    out = []
    for k, (nemd, grd) in enumerate(gold["emit_faces"]):
        nemd = int(nemd)
        b1, b2 = tang[abs(nemd)]
        uu = u[k * 6 * n:(k + 1) * 6 * n].reshape(n, 6)
        out.append(inject.emit_plane(nemd, float(grd), b1, b2, n, gold["emit_vnormf"], gold["emit_vtangf"], injctisw,
                                     None, spec=1, uniforms=uu))
    got = np.concatenate(out)
    want = gold["emit_records"]
    assert got.size == want.size
    for f in KIN:
        assert np.array_equal(got[f], want[f]), f


def test_emission_pairs(gold):
    """psuper3's emission pairs (emit_from_rectangle, psuper3.F90:142-208):
    an anti-particle on the face and its twin 1e-5 off it, per face."""
    n = int(gold["emit_n"])
    xl, xu, yl, yu, zl, zu = gold["emit_bounds"]
    tang = {1: ((yl, yu), (zl, zu)), 2: ((zl, zu), (xl, xu)), 3: ((xl, xu), (yl, yu))}
    u = gold["pair_uniforms"]
    out = []
    for k, (nemd, grd) in enumerate(gold["emit_faces"]):
        nemd = int(nemd)
        b1, b2 = tang[abs(nemd)]
        uu = u[k * 6 * n:(k + 1) * 6 * n].reshape(n, 6)
        out.append(inject.emit_rectangle(nemd, float(grd), b1, b2, n, gold["emit_vnormf"], gold["emit_vtangf"], None,
                                         spec=1, uniforms=uu))
    got = np.concatenate(out)
    want = gold["pair_records"]
    assert got.size == want.size == 2 * n * len(gold["emit_faces"])
    for f in KIN + ("preside", "spec", "pid"):
        assert np.array_equal(got[f], want[f]), f


def test_emission_count(gold):
    """nemit of psuper3.F90:68-69 over steps, step offsets, intervals,
    fluxes and ustep."""
    for istep, lstep, injct, fluxf, ustep, n in gold["count_rows"]:
        assert inject.emission_count(int(istep), int(lstep), fluxf, int(injct), int(ustep)) == int(n)


def test_cylinder_emission(gold):
    """psuper3's emission from cylinders (emit_from_cylinder with
    emit_from_circular_surf and emit_from_cylindrical_surf1/2/3,
    psuper3.F90:241-528): end caps and side surfaces of cylinders along x, y
    and z, the three side kinds (radius >= 1, radius < 1 with five uniforms a
    particle, omnidirectional), with and without anti-particles."""
    n = int(gold["cyl_n"])
    xl, xu, yl, yu, zl, zu = gold["cyl_bounds"]
    psixy, psizx, psizy = gold["cyl_psi"]
    along = {1: (xl, xu, psizy), 2: (yl, yu, psizx), 3: (zl, zu, psixy)}
    tabs = {k: gold["cyl_" + k] for k in ("vnormf", "vtangf", "runiform", "vnormc", "vtangc", "psicos")}
    u = gold["cyl_uniforms"]
    out = []
    for k, (align, radius, omni, ncond, nemd, grd) in enumerate(gold["cyl_cases"]):
        hl, hu, psi = along[int(align)]
        out.append(inject.emit_cylinder(int(nemd), int(align), radius, tuple(gold["cyl_axis"]), int(omni), grd, hl,
                                        hu, psi, n, tabs, None, spec=1, uniforms=u[k * 6 * n:(k + 1) * 6 * n],
                                        anti=int(ncond) <= 0))
    got = np.concatenate(out)
    want = gold["cyl_records"]
    assert got.size == want.size
    for f in KIN + ("preside", "spec", "pid", "nid"):
        assert np.array_equal(got[f], want[f]), f


def test_psuper1_inflow_current(gold):
    """psuper1's outer-face inflow with its injection current
    (psuper1.F90:120-323, current_deposition :859-988): the records of the
    six faces and the zigzag current of every particle's path from outside
    the face to its injection point, bit for bit."""
    nx, ny, nz = (int(v) for v in gold["p1_ext"])
    npr, ustep, injct, istep, lstep = (int(v) for v in gold["p1_setup"])
    t = {k[7:]: gold[k] for k in gold if k.startswith("p1_tab_")}
    faces = [("arrxf", 0, True, t["vxf"], t["vyr"], t["vzr"]), ("arrxb", 0, False, t["vxb"], t["vyr"], t["vzr"]),
             ("arryf", 1, True, t["vyf"], t["vxr"], t["vzr"]), ("arryb", 1, False, t["vyb"], t["vxr"], t["vzr"]),
             ("arrzf", 2, True, t["vzf"], t["vxr"], t["vyr"]), ("arrzb", 2, False, t["vzb"], t["vxr"], t["vyr"])]
    u = gold["p1_uniforms"]
    pos = 0
    recs = []
    wrk = np.zeros((nz + 9, ny + 9, nx + 9, 3))
    for key, axis, front, vn, va, vb in faces:
        n = inject.inflow_count(istep, lstep, float(gold["p1_arr_" + key]), injct, ustep)
        assert n == int(gold["p1_count_" + key]), key
        r = inject.inflow(axis, front, n, nx, ny, nz, vn, va, vb, float(injct * ustep), None, spec=1,
                          uniforms=u[pos:pos + 5 * n].reshape(n, 5))
        pos += 5 * n
        inject.inflow_current(axis, front, r, ustep, (nx, ny, nz), wrk)
        recs.append(r)
    assert pos == u.size
    got = np.concatenate(recs)
    want = gold["p1_records"]
    assert got.size == want.size > 0
    for f in KIN + ("preside", "spec"):
        assert np.array_equal(got[f], want[f]), f
    # the fixture's wrk is (3, x, y, z) over the nodes -4..n+4
    ref = np.transpose(gold["p1_wrk"], (3, 2, 1, 0))
    assert np.count_nonzero(ref) > 0
    assert np.array_equal(wrk.view(np.uint64), np.ascontiguousarray(ref).view(np.uint64))
