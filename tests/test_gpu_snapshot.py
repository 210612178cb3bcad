"""A restart through the esdat snapshot: the FP32 form's state after some
steps is written (ctca_b200.snapshot.save), a new context starts from the
file, and its particles equal the first context's bit for bit (as a set:
the restart re-sorts them); the next step of both gives the same rho and J
up to the FP32 run sums' order (1e-6)."""
import numpy as np
import pytest

from ctca_b200 import inputs, snapshot
from ctca_b200.emses import Emses
from oracle import compare as C

pytestmark = pytest.mark.gpu


def as_set(p):
    live = p[p["nid"] != -1]
    return live[np.lexsort([live[f] for f in ("vz", "vy", "vx", "z", "y", "x", "spec")])]


def test_restart_through_esdat(gpu, tmp_path):
    case = inputs.workload_case(2, scale=0.125)
    for s in case.species:
        s.ppc = 8
    cfg = inputs.make_config(case)
    eb = inputs.make_fields(case)
    u = inputs.units()
    rens = (1.0, u["renv"], u["renrho"], u["renq"])
    path = tmp_path / snapshot.esdat_name(0)
    with Emses(cfg) as g:
        g.upload_field("eb", eb)
        g.load_plasma(inputs.plasma(case))
        g.fx_load()
        for s in range(3):
            g.fx_step(2, s == 1)
        snapshot.save(g, path, rens)
        first, tp1 = g.download_particles()
        g.fx_step(2, False)
        rho1, aj1 = g.download_field("rho"), g.download_field("aj")
    with Emses(cfg) as h:
        h.upload_field("eb", eb)
        d = snapshot.load(h, path)
        assert np.array_equal(d["totalp"], tp1[:cfg.nspec])
        assert np.array_equal(d["rens"], np.array(rens))
        h.fx_store()
        back, tp2 = h.download_particles()
        assert np.array_equal(tp2, tp1)
        a, b = as_set(first), as_set(back)
        for f in ("x", "y", "z", "vx", "vy", "vz", "spec"):
            assert np.array_equal(a[f], b[f]), f
        h.fx_load()
        h.fx_step(2, False)
        assert C.field_errors(h.download_field("rho"), rho1, cfg)["l2_rel"] < 1e-6
        assert C.field_errors(h.download_field("aj"), aj1, cfg)["l2_rel"] < 1e-6
