"""The oracle against the golden fixtures of tests/golden/: outputs of the
reference's own Fortran subroutines (grdcrt, psolve2, psolve1,
add_boundary_current(2), charge, add_boundary_charge, rhoupd, positn,
bfield, efield), executed from their source text by
tests/golden/make_golden.py on small seeded cases.

Every comparison is bit-for-bit: particles (all 64 bytes of each record),
every field element, every counter, and the number of random numbers drawn.
"""
from pathlib import Path

import numpy as np
import pytest

from ctca_b200.emses import Config
from oracle import oracle as O

# the particle-path fixtures of make_golden.py (supervisors.npz and
# tables.npz, of make_golden_supervisors.py and make_golden_tables.py, have
# their own tests)
CASES = sorted(p for p in (Path(__file__).parent / "golden").glob("*.npz") if p.stem not in ("supervisors", "tables"))


def load(path):
    d = dict(np.load(path))
    cfg = Config.from_buffer_copy(d["config"].tobytes())
    cfg.rng_mode = 1  # RANU0 draws come from the fixture's list of uniforms
    return d, cfg


def oracle_for(d, cfg, pbuf):
    o = O.Oracle(cfg, pbuf, d["totalp"], d["eb"])
    o.set_randoms(d["uniforms"])
    return o


def same(a, b):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def first_diff(a, b):
    idx = np.argwhere(a != b)
    return f"{len(idx)} differ, first at {tuple(idx[0])}: {a[tuple(idx[0])]!r} vs {b[tuple(idx[0])]!r}" if len(idx) else ""


def check_counters(o, d, prefix):
    got = o.gc.as_dict()
    for k in ("influx", "infhist", "nesc", "chgacm"):
        assert same(got[k].astype(d[prefix + k].dtype), d[prefix + k]), (k, first_diff(got[k], d[prefix + k]))


def test_fixtures_present():
    assert {p.stem for p in CASES} >= {"periodic", "walls", "walls_z", "bodies"}


@pytest.mark.parametrize("path", CASES, ids=lambda p: p.stem)
def test_grdcrt_and_psolve2(path):
    d, cfg = load(path)
    o = oracle_for(d, cfg, d["pbuf0"])
    o.grdcrt()
    assert same(o.f["wrk"], d["wrk"]), first_diff(o.f["wrk"], d["wrk"])
    o.psolve2(int(d["ustep"]))
    assert o.ranu_pos.value == int(d["psolve2_nranu"])
    for fld in d["pbuf0"].dtype.names:
        assert same(o.pbuf[fld], d["psolve2_pbuf"][fld]), (fld, first_diff(o.pbuf[fld], d["psolve2_pbuf"][fld]))
    check_counters(o, d, "psolve2_")


@pytest.mark.parametrize("path", CASES, ids=lambda p: p.stem)
def test_psolve1_charge_and_reductions(path):
    d, cfg = load(path)
    o = oracle_for(d, cfg, d["pbuf0"])
    o.grdcrt()
    o.psolve1(int(d["ustep"]), 1)
    assert o.ranu_pos.value == int(d["psolve1_nranu"])
    for fld in d["pbuf0"].dtype.names:
        assert same(o.pbuf[fld], d["psolve1_pbuf"][fld]), (fld, first_diff(o.pbuf[fld], d["psolve1_pbuf"][fld]))
    check_counters(o, d, "psolve1_")
    assert np.abs(d["psolve1_aj"]).max() > 0
    assert same(o.f["aj"], d["psolve1_aj"]), first_diff(o.f["aj"], d["psolve1_aj"])
    assert same(o.f["ajdg"], d["psolve1_ajdg"]), first_diff(o.f["ajdg"], d["psolve1_ajdg"])
    o.reduce_aj()
    assert same(o.f["aj"], d["reduced_aj"]), first_diff(o.f["aj"], d["reduced_aj"])
    o.reduce_ajdg()
    assert same(o.f["ajdg"], d["reduced_ajdg"]), first_diff(o.f["ajdg"], d["reduced_ajdg"])

    o.pbuf = d["charge_pbuf_in"].copy()
    o.charge(2)
    assert same(o.pbuf, d["charge_pbuf"])
    for nm in ("rho", "rhodg", "rhobk", "rhobksp"):
        assert same(o.f[nm], d["charge_" + nm]), (nm, first_diff(o.f[nm], d["charge_" + nm]))
    assert np.abs(d["charge_rhobk"]).max() > 0
    o.reduce_rho("rho")
    assert same(o.f["rho"], d["reduced_rho"]), first_diff(o.f["rho"], d["reduced_rho"])
    o.reduce_rho("rhodg")
    assert same(o.f["rhodg"], d["reduced_rhodg"]), first_diff(o.f["rhodg"], d["reduced_rhodg"])
    o.rhoupd()
    assert same(o.f["rho"], d["rhoupd_rho"]), first_diff(o.f["rho"], d["rhoupd_rho"])


@pytest.mark.parametrize("path", CASES, ids=lambda p: p.stem)
def test_positn(path):
    d, cfg = load(path)
    o = oracle_for(d, cfg, d["pbuf0"])
    o.positn(int(d["ustep"]))
    assert o.ranu_pos.value == int(d["positn_nranu"])
    for fld in d["pbuf0"].dtype.names:
        assert same(o.pbuf[fld], d["positn_pbuf"][fld]), (fld, first_diff(o.pbuf[fld], d["positn_pbuf"][fld]))
    check_counters(o, d, "positn_")


@pytest.mark.parametrize("path", CASES, ids=lambda p: p.stem)
def test_field_step(path):
    """bfield, efield (with the reduced aj) and the eb border exchange."""
    d, cfg = load(path)
    o = oracle_for(d, cfg, d["pbuf0"])
    o.bfield()
    assert same(o.eb, d["bfield_eb"]), first_diff(o.eb, d["bfield_eb"])
    o.f["aj"][...] = d["reduced_aj"]
    o.efield(float(d["tcs"]))
    assert same(o.eb, d["efield_eb"]), first_diff(o.eb, d["efield_eb"])
    o.exchange_eb()
    assert same(o.eb, d["exchange_eb"]), first_diff(o.eb, d["exchange_eb"])


@pytest.mark.parametrize("path", CASES, ids=lambda p: p.stem)
def test_energy(path):
    """Kinetic energy per species and axis (energy.F90:29-47) of the state
    after positn, bit for bit."""
    d, cfg = load(path)
    o = oracle_for(d, cfg, d["positn_pbuf"].copy())
    e = o.energy().reshape(cfg.nspec, 3).T
    want = d["energy_engk"]
    assert same(e, want), first_diff(e, want)
