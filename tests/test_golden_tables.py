"""ctca_b200.tables against the reference's table code executed from its
own text with its own random stream (tests/golden/make_golden_tables.py):
bit for bit."""
from pathlib import Path

import numpy as np
import pytest

from ctca_b200 import tables as T

G = np.load(Path(__file__).parent / "golden" / "tables.npz")


def same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.uint64) if a.dtype == np.float64 else a,
                                                 b.view(np.uint64) if b.dtype == np.float64 else b)


def test_stream_is_the_reference_mersenne_twister():
    r = T.Ranu0(int(G["stream_seed"][0]))
    assert same(r.draw(1000), G["stream"][:1000])
    assert same(r.draw(G["stream"].size - 1000), G["stream"][1000:])


@pytest.mark.parametrize("c", range(7))
def test_vflux(c):
    na, v0, vt, isl, seed, icon, used = G["vflux_cases"][c]
    r = T.Ranu0(int(seed))
    t, ic = T.vflux(int(na), v0, vt, int(isl), r)
    assert same(t, G[f"vflux_{c}"])
    assert ic == int(icon) and r.drawn == int(used)


@pytest.mark.parametrize("c", range(5))
def test_vinit(c):
    na, v0, vt, xlos, seed, v0o, vto, used = G["vinit_cases"][c]
    r = T.Ranu0(int(seed))
    t, v0n, vtn = T.vinit(int(na), v0, vt, xlos, r)
    assert same(t, G[f"vinit_{c}"])
    assert v0n == v0o and vtn == vto and r.drawn == int(used)


@pytest.mark.parametrize("c", range(2))
def test_ringds(c):
    na, vt, bbb, seed, used = G["ringds_cases"][c]
    r = T.Ranu0(int(seed))
    assert same(T.ringds(int(na), vt, bbb, r), G[f"ringds_{c}"])
    assert r.drawn == int(used)


@pytest.mark.parametrize("c", range(3))
def test_rann0(c):
    am, sd, n, seed, used = G["rann0_cases"][c]
    r = T.Ranu0(int(seed))
    assert same(T.rann0(am, sd, int(n), r), G[f"rann0_{c}"])
    assert r.drawn == int(used)


def test_rexch_same_pairs_in_every_array():
    n, seed, used = (int(x) for x in G["rexch_case"])
    i1 = np.arange(1, n + 1, dtype=np.int64)
    d1 = np.arange(n, dtype=np.float64) * 0.5
    d5 = -np.arange(n, dtype=np.float64)
    r = T.Ranu0(seed)
    T.rexch(n, [i1, d1, d5], r)
    assert np.array_equal(i1, G["rexch_i1"]) and same(d1, G["rexch_d1"]) and same(d5, G["rexch_d5"])
    assert r.drawn == used


def test_inflow_tables_two_species():
    """The outer-boundary tables of inipin for two species in one stream,
    the second with nphi = 2, and the inflow rates."""
    seed, used = (int(x) for x in G["inflow_case"])
    slx, sly, slz, ex, ey, ez, dt = G["inflow_grid"]
    r = T.Ranu0(seed)
    o = 0
    for s, (npr, nphi, vdx, vdy, vdz, peth, path, npin) in enumerate(G["inflow_species"]):
        npr = int(npr)
        tb = T.inflow_tables(npr, int(nphi), (vdx, vdy, vdz), peth, path, r)
        for k in ("vxf", "vyf", "vzf", "vxb", "vyb", "vzb", "vxr", "vyr", "vzr"):
            assert same(tb[k], G[f"inflow_{k}"][o:o + npr]), (s, k)
        rates = T.inflow_rates((vdx, vdy, vdz), peth, path, npin, (slx, sly, slz), (ex, ey, ez), dt)
        for k, v in rates.items():
            assert v == G[f"inflow_{k}"][s], (s, k)
        o += npr
    assert r.drawn == used


@pytest.mark.parametrize("variant", (0, 1))
def test_emission_tables_two_species(variant):
    """assign_velocity for two species in one stream (variant 1: second
    populations in the flux and tangential tables)."""
    seed, used, path2, peth2, mainprop = G[f"emit{variant}_case"]
    r = T.Ranu0(int(seed))
    vxf = G["emit_vxf"]
    o = 0
    for s, (npr, nphi, spa, abvdem, spe, peth, path) in enumerate(G["emit_species"]):
        npr = int(npr)
        npq = npr // int(nphi)
        tb = T.emission_tables(npr, npq, spa + abvdem, path, peth, spe, r, vxf=vxf[o:o + npr], path2=path2,
                               peth2=peth2, mainprop=mainprop)
        for k in ("vnormf", "vtangf", "runiform", "vnormc", "vtangc", "psicos", "vnorms", "vtangs1", "vtangs2"):
            assert same(tb[k], G[f"emit{variant}_{k}"][o:o + npr]), (s, k)
        o += npr
    assert r.drawn == int(used)
