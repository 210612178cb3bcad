"""The GPU adjoint (emsesg_fx_adjoint: FP32 reverse sweep with checkpoints
and recompute, through the re-sorts) against the FP64 CPU adjoint of the
oracle (oracle/adjoint.cpp, itself checked against central differences) on
the same FP32-rounded start state and node fields.

Tolerances: loss 1e-5 relative; gradients 2e-3 relative L2 (FP32
trajectories and FP32 gradient sums against FP64)."""
import numpy as np
import pytest

from ctca_b200.emses import Emses
from oracle import oracle as O

from helpers import build, case, rel_l2

pytestmark = pytest.mark.gpu


def node_fields(cfg, o):
    """FP32 node fields of the push (grdcrt) split into node part + e0/b0."""
    o.grdcrt()
    w = o.f["wrk"]
    nx, ny, nz = cfg.nx, cfg.ny, cfg.nz
    nodes = w[4:4 + nz, 4:4 + ny, 4:4 + nx, :6].astype(np.float32).astype(np.float64)
    e0b0 = np.array(list(cfg.e0) + list(cfg.b0))
    en = (nodes[..., :3] - e0b0[:3]).reshape(-1, 3)   # x fastest: (k, j, i) C order
    bn = (nodes[..., 3:6] - e0b0[3:]).reshape(-1, 3)
    return en, bn, e0b0


@pytest.mark.parametrize("K,ckpt,sort_every", [(8, 4, 4), (6, 2, 3)])
def test_gpu_adjoint_matches_fp64_adjoint(gpu, K, ckpt, sort_every):
    c = case(n=(16, 16, 16), ppc=(2, 2), seed=21, b0=(0.05, -0.1, 0.2), vth_scale=2.0, tile=(8, 8, 8))
    cfg, eb, p, tp = build(c)
    g = Emses(cfg)
    g.upload_particles(p, tp)
    g.upload_field("eb", eb)
    g.fx_load()
    g.fx_store()
    p32, tp32 = g.download_particles()
    g.fx_load()
    o = O.Oracle(cfg, p32, tp32, eb)
    en, bn, e0b0 = node_fields(cfg, o)
    lo, hi = (4, 4, 4), (12, 12, 12)
    loss_o, gE_o, gB_o, g0_o, gv_o = O.adjoint(cfg, K, 2, en, bn, e0b0, p32, lo, hi)
    loss, gE, gB, g0, gv = g.fx_adjoint(K, 2, ckpt, sort_every, lo, hi, int(tp32.sum()))
    g.close()
    assert loss_o > 0
    assert abs(loss - loss_o) <= 1e-5 * loss_o
    assert rel_l2(g0, g0_o) < 2e-3
    assert rel_l2(gE, gE_o) < 2e-3
    assert rel_l2(gB, gB_o) < 2e-3
    assert rel_l2(gv, gv_o) < 2e-3
