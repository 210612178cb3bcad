"""The FP64 GPU drop-in against the golden fixtures made from the reference's
own Fortran source (tests/golden/), through the C ABI.

Particle records, counters and the number of random numbers drawn must be
bit-identical; fields formed by FP64 atomics (J, rho) agree to 1e-12
relative L2, the summation-order tolerance; grdcrt is bit-identical."""
import numpy as np
import pytest

from ctca_b200.emses import Config, Counter, Emses

from helpers import rel_l2, same_particles
from test_golden import CASES

pytestmark = pytest.mark.gpu

TOL = 1e-12


def load(path):
    d = dict(np.load(path))
    cfg = Config.from_buffer_copy(d["config"].tobytes())
    cfg.rng_mode = 1
    return d, cfg


def device(d, cfg, pbuf):
    g = Emses(cfg)
    g.upload_particles(pbuf, d["totalp"])
    g.upload_field("eb", d["eb"])
    g.set_randoms(d["uniforms"])
    return g


def counters_match(gc: Counter, d, prefix):
    got = gc.as_dict()
    for k in ("influx", "infhist", "nesc", "chgacm"):
        assert np.array_equal(got[k].astype(d[prefix + k].dtype), d[prefix + k]), k


@pytest.mark.parametrize("path", CASES, ids=lambda p: p.stem)
def test_dropin_grdcrt_psolve2_golden(gpu, path):
    d, cfg = load(path)
    with device(d, cfg, d["pbuf0"]) as g:
        g.grdcrt(1)
        w = g.download_field("wrk")
        assert np.array_equal(w[..., :6], d["wrk"][..., :6])
        gc = Counter()
        g.psolve2(1, int(d["ustep"]), gc)
        p, tp = g.download_particles()
        assert np.array_equal(tp, d["totalp"])
        assert same_particles(p, d["psolve2_pbuf"])
        counters_match(gc, d, "psolve2_")


@pytest.mark.parametrize("path", CASES, ids=lambda p: p.stem)
def test_dropin_psolve1_charge_golden(gpu, path):
    d, cfg = load(path)
    with device(d, cfg, d["pbuf0"]) as g:
        g.grdcrt(1)
        g.zero_field("aj")
        g.zero_field("ajdg")
        gc = Counter()
        g.psolve1(1, int(d["ustep"]), 1, gc)
        p, _ = g.download_particles()
        assert same_particles(p, d["psolve1_pbuf"])
        counters_match(gc, d, "psolve1_")
        assert rel_l2(g.download_field("aj"), d["psolve1_aj"]) < TOL
        assert rel_l2(g.download_field("ajdg"), d["psolve1_ajdg"]) < TOL
        g.reduce_aj()
        g.reduce_ajdg()
        assert rel_l2(g.download_field("aj"), d["reduced_aj"]) < TOL
        assert rel_l2(g.download_field("ajdg"), d["reduced_ajdg"]) < TOL
        g.upload_particles(d["charge_pbuf_in"], d["totalp"])
        for nm in ("rho", "rhodg", "rhobk", "rhobksp"):
            g.zero_field(nm)
        g.charge(1, 2)
        p, _ = g.download_particles()
        assert same_particles(p, d["charge_pbuf"])
        for nm in ("rho", "rhodg", "rhobk", "rhobksp"):
            assert rel_l2(g.download_field(nm), d["charge_" + nm]) < TOL, nm
        g.reduce_rho("rho")
        g.reduce_rho("rhodg")
        assert rel_l2(g.download_field("rho"), d["reduced_rho"]) < TOL
        assert rel_l2(g.download_field("rhodg"), d["reduced_rhodg"]) < TOL
        g.rhoupd(1)
        assert rel_l2(g.download_field("rho"), d["rhoupd_rho"]) < TOL


@pytest.mark.parametrize("path", CASES, ids=lambda p: p.stem)
def test_dropin_positn_golden(gpu, path):
    d, cfg = load(path)
    with device(d, cfg, d["pbuf0"]) as g:
        gc = Counter()
        g.positn(1, int(d["ustep"]), gc)
        p, _ = g.download_particles()
        assert same_particles(p, d["positn_pbuf"])
        counters_match(gc, d, "positn_")


@pytest.mark.parametrize("path", CASES, ids=lambda p: p.stem)
def test_dropin_field_step_golden(gpu, path):
    d, cfg = load(path)
    with device(d, cfg, d["pbuf0"]) as g:
        g.bfield(1)
        assert np.array_equal(g.download_field("eb"), d["bfield_eb"])
        g.upload_field("aj", d["reduced_aj"])
        g.efield(1, float(d["tcs"]))
        assert np.array_equal(g.download_field("eb"), d["efield_eb"])
        g.exchange_eb()
        assert np.array_equal(g.download_field("eb"), d["exchange_eb"])
