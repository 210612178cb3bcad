"""The FP64 CPU adjoint of the periodic push + zigzag current (oracle/
adjoint.cpp) against central finite differences of its own forward loss.

The zigzag J jumps by the cubic term q*dx*dy*dz/8 when a particle's end
point crosses a cell face (the relay point moves from the midpoint to the
face), so the loss is piecewise smooth; the differences use steps small
enough (1e-7 relative) that no particle crosses a face within them."""
import numpy as np
import pytest

from ctca_b200 import inputs
from oracle import oracle as O

from helpers import case


@pytest.fixture(scope="module")
def problem():
    c = case(n=(8, 8, 8), ppc=(2, 2), seed=5, b0=(0.05, -0.1, 0.2))
    cfg = inputs.make_config(c)
    p, _ = inputs.make_particles(c)
    rng = np.random.default_rng(0)
    en = rng.normal(0, 1e-3, (512, 3))
    bn = rng.normal(0, 2e-2, (512, 3))
    e0 = np.array([1e-3, -5e-4, 2e-4, 0.01, -0.02, 0.05])
    args = dict(K=4, lo=(2, 2, 2), hi=(6, 6, 6))
    loss, gE, gB, g0, gv = O.adjoint(cfg, args["K"], 2, en, bn, e0, p, args["lo"], args["hi"])
    return cfg, p, en, bn, e0, args, (loss, gE, gB, g0, gv)


def L(cfg, args, en, bn, e0, p):
    return O.adjoint(cfg, args["K"], 2, en, bn, e0, p, args["lo"], args["hi"], grad=False)[0]


def rel(a, b):
    return abs(a - b) / max(abs(a), abs(b), 1e-300)


def test_background_field_gradients(problem):
    cfg, p, en, bn, e0, args, (loss, gE, gB, g0, gv) = problem
    assert loss > 0
    for k in range(6):
        h = 1e-7 * max(abs(e0[k]), 1e-3)
        a, b = e0.copy(), e0.copy()
        a[k] += h
        b[k] -= h
        fd = (L(cfg, args, en, bn, a, p) - L(cfg, args, en, bn, b, p)) / (2 * h)
        assert rel(g0[k], fd) < 1e-5, (k, g0[k], fd)
    # e0/b0 act as a uniform node field: their gradients are the node sums
    assert np.allclose(g0[:3], gE.sum(axis=0), rtol=1e-10, atol=0)
    assert np.allclose(g0[3:], gB.sum(axis=0), rtol=1e-10, atol=0)


def test_node_field_gradients(problem):
    cfg, p, en, bn, e0, args, (loss, gE, gB, g0, gv) = problem
    rng = np.random.default_rng(1)
    nodes = rng.choice(np.flatnonzero(np.abs(gE).sum(axis=1) > 0), 6, replace=False)
    for node in nodes:
        for comp in range(3):
            for arr, g in ((en, gE), (bn, gB)):
                h = 1e-8
                a, b = arr.copy(), arr.copy()
                a[node, comp] += h
                b[node, comp] -= h
                ea, eb_ = (a, b) if arr is en else (en, en)
                ba, bb = (a, b) if arr is bn else (bn, bn)
                fd = (L(cfg, args, ea, ba, e0, p) - L(cfg, args, eb_, bb, e0, p)) / (2 * h)
                # central differences carry ~eps*L/h of rounding
                assert abs(g[node, comp] - fd) <= 1e-4 * abs(fd) + 1e-16 * loss / h * 50, (node, comp)


def test_initial_velocity_gradients(problem):
    cfg, p, en, bn, e0, args, (loss, gE, gB, g0, gv) = problem
    rng = np.random.default_rng(2)
    ms = rng.choice(np.flatnonzero(np.abs(gv).sum(axis=1) > 0), 8, replace=False)
    for m in ms:
        for comp, f in enumerate(("vx", "vy", "vz")):
            h = 1e-9
            a, b = p.copy(), p.copy()
            a[f][m] += h
            b[f][m] -= h
            fd = (L(cfg, args, en, bn, e0, a) - L(cfg, args, en, bn, e0, b)) / (2 * h)
            assert abs(gv[m, comp] - fd) <= 1e-4 * abs(fd) + 1e-16 * loss / h * 50, (m, comp)


def test_checkpointed_adjoint_equals_the_full_one(problem):
    """Keeping the state every 2 steps and recomputing in between gives the
    same loss and gradients, bit for bit."""
    cfg, p, en, bn, e0, args, (loss, gE, gB, g0, gv) = problem
    r = O.adjoint(cfg, args["K"], 2, en, bn, e0, p, args["lo"], args["hi"], ckpt=2)
    assert r[0] == loss
    for a, b in zip(r[1:], (gE, gB, g0, gv)):
        assert np.array_equal(a, b)
