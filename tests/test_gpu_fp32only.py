"""FP32-only contexts (EMSESG_FLAG_FP32_ONLY) and the direct FP32 plasma
loader (emsesg_fx_load_plasma).

emsesg_fx_load_plasma draws the same particles as emsesg_load_plasma and
converts them with the same kernel as emsesg_fx_load, so the two routes give
bit-identical particle states and bit-identical int64 rho/J accumulators
after a few steps.  A context without the FP64 particle buffer refuses the
calls that move FP64 records."""
import numpy as np
import pytest

from ctca_b200 import inputs
from ctca_b200.emses import Emses, EmsesError

from helpers import case

pytestmark = pytest.mark.gpu

FP32_ONLY = 1


def setup(c, flags=0):
    cfg = inputs.make_config(c)
    cfg.flags = flags
    g = Emses(cfg)
    g.upload_field("eb", inputs.make_fields(c))
    return g


def test_fx_load_plasma_matches_load_plasma_then_fx_load(gpu):
    c = case(n=(16, 16, 24), ppc=(7, 5), tile=(8, 8, 8))
    pl = inputs.plasma(c, seed=123)
    with setup(c) as a, setup(c) as b:
        a.load_plasma(pl)
        a.fx_load()
        b.fx_load_plasma(pl)
        assert np.array_equal(a.fx_counts(), b.fx_counts())
        a.fx_store()
        b.fx_store()
        pa, ta = a.download_particles()
        pb, tb = b.download_particles()
        assert np.array_equal(ta, tb)
        assert np.array_equal(pa.view(np.uint8), pb.view(np.uint8))


def test_fp32_only_context_steps_like_a_full_one(gpu):
    c = case(n=(16, 16, 16), ppc=(6, 6), tile=(8, 8, 8), vth_scale=2.0)
    pl = inputs.plasma(c, seed=7)
    with setup(c) as a, setup(c, FP32_ONLY) as b:
        a.load_plasma(pl)
        a.fx_load()
        b.fx_load_plasma(pl)
        for s in range(6):
            a.fx_step(2, s % 3 == 2)
            b.fx_step(2, s % 3 == 2)
        a.synchronize()
        b.synchronize()
        ra, ja = a.fx_download_accum()
        rb, jb = b.fx_download_accum()
        assert np.array_equal(ra, rb)
        assert np.array_equal(ja, jb)
        assert np.array_equal(a.fx_counts(), b.fx_counts())
        assert np.array_equal(a.download_field("rho"), b.download_field("rho"))


def test_fp32_only_context_refuses_fp64_records(gpu):
    c = case(n=(8, 8, 8), ppc=(2, 2))
    cfg, eb = inputs.make_config(c), inputs.make_fields(c)
    p, tp = inputs.make_particles(c)
    with setup(c, FP32_ONLY) as g:
        with pytest.raises(EmsesError, match="FP32-only"):
            g.upload_particles(p, tp)
        with pytest.raises(EmsesError, match="FP32-only"):
            g.load_plasma(inputs.plasma(c))
        with pytest.raises(EmsesError, match="FP32-only"):
            g.fx_load()
        g.fx_load_plasma(inputs.plasma(c))
        with pytest.raises(EmsesError, match="FP32-only"):
            g.fx_store()
        with pytest.raises(EmsesError, match="FP32-only"):
            g.download_particles()
