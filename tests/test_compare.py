"""The checker's helpers (oracle/compare.py) import and run on CPU data, so
that a GPU test never meets a missing one."""
import numpy as np

from ctca_b200 import inputs
from oracle import compare as C


def test_helpers_on_cpu_data():
    case = inputs.workload_case(1)
    case.n = (8, 8, 8)
    cfg = inputs.make_config(case)
    p, tp = inputs.make_particles(case)
    rep = C.particle_errors(cfg, p, p.copy())
    assert rep["cell_mismatch"] == 0 and rep["pos_max_abs"] == 0.0 and len(rep["mismatched"]) == 0
    rho = np.random.default_rng(0).random((11, 11, 11, 1))
    aj = np.random.default_rng(1).random((17, 17, 17, 3))
    assert C.nodes(cfg, rho).shape == (9, 9, 9, 1) and C.nodes(cfg, aj).shape == (9, 9, 9, 3)
    assert C.field_errors(rho, rho, cfg)["l2_rel"] == 0.0
    assert C.j_error_corrected(cfg, aj, aj, p, p, p, [])[1] == 0.0
    key, tid = C.tile_key(cfg, (4, 4, 4), p)
    assert key.shape == tid.shape == (p.size,)
    order = C.sort_order(cfg, (4, 4, 4), 736, p[:tp[0]], p[:tp[0]])
    assert sorted(order) == list(range(tp[0]))
    assert C.cell_histogram(cfg, p).sum() == p.size
    assert C.continuity_residual(cfg, rho, rho, np.zeros_like(aj)) == 0.0
    assert not C.near_faces(cfg, p, p).all()
