"""The timed CPU baseline (oracle/baseline.cpp): the reference's one rank
per core, each thread owning a block of x rows with its own sub-grid, must
give the particles, aj and rho of the single-threaded oracle (psolve1 +
add_boundary_current, charge + add_boundary_charge) on a periodic grid, for
the whole grid and for a sample of z layers; a second step starts again
from the initial particles."""
import numpy as np
import pytest

from ctca_b200 import inputs
from oracle import oracle as O

from helpers import rel_l2


def interior(cfg, name, a):
    lo = -4 if name == "aj" else -1
    return a[-lo:-lo + cfg.nz, -lo:-lo + cfg.ny, -lo:-lo + cfg.nx]


@pytest.mark.parametrize("threads,layers", [(1, None), (3, None), (4, (2, 5)), (7, (0, 8))])
def test_blocks_match_the_oracle(threads, layers):
    case = inputs.workload_case(2)
    case.n = (8, 12, 8)
    case.kmax = 2 * np.pi / 4
    for s in case.species:
        s.ppc = 3
    cfg = inputs.make_config(case)
    eb = inputs.make_fields(case)
    p, tp = inputs.make_particles(case)
    if layers:
        keep = (np.floor(p["z"]) >= layers[0]) & (np.floor(p["z"]) < layers[1])
        p = np.concatenate([p[: tp[0]][keep[: tp[0]]], p[tp[0]:][keep[tp[0]:]]])
        tp = np.array([keep[: tp[0]].sum(), keep[tp[0]:].sum()])
    o = O.Oracle(cfg, p, tp, eb)
    o.grdcrt()
    b = O.Blocks(cfg, o.f["wrk"], p, tp, threads)
    assert b.particles == int(tp.sum())
    assert 1 <= b.threads <= threads
    for _ in range(2):  # every step starts from the given particles
        assert b.step(2) >= 0.0
    aj, rho = b.result()
    o.f["aj"][...] = 0.0
    o.psolve1(2, 0)
    o.reduce_aj()
    o.charge(0)
    o.reduce_rho("rho")
    assert rel_l2(interior(cfg, "aj", aj), interior(cfg, "aj", o.f["aj"])) < 1e-13
    assert rel_l2(interior(cfg, "rho", rho), interior(cfg, "rho", o.f["rho"])) < 1e-13
    b.close()
