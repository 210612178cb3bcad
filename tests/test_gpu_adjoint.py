"""The GPU adjoint (emsesg_fx_adjoint: FP32 reverse sweep with checkpoints
and recompute, through the re-sorts, FP64 sums of the node-field gradients)
against the FP64 CPU adjoint of the oracle (oracle/adjoint.cpp, itself
checked against central differences) and against central finite
differences of the FP64 forward loss, on the same FP32-rounded start state
and node fields.

Tolerances: loss 1e-5 relative; gradients 1e-5 relative L2 against the FP64
adjoint for K <= 8, 1e-4 per parameter against central differences.  The
loss is piecewise smooth (the zigzag current jumps when an end point crosses
a cell face), so each difference uses the largest relative step of 1e-3,
1e-4, 1e-5, 1e-6 at which it is stable (the next smaller step gives the same
difference to 1e-5): a step that moves an end point across a face measures
the jump, not the derivative."""
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
    for a, b in ((g0, g0_o), (gE, gE_o), (gB, gB_o), (gv, gv_o)):
        assert rel_l2(a, b) < 1e-5


def fd_derivative(f, theta, scale):
    """Central difference of f at theta with the largest relative step of
    1e-3 .. 1e-6 (times scale) that agrees with the next smaller one to 1e-5
    (no face crossed); returns (derivative, step)."""
    prev = None
    steps = (1e-3, 1e-4, 1e-5, 1e-6, 1e-7)
    vals = []
    for s in steps:
        h = s * scale
        vals.append(((f(theta + h) - f(theta - h)) / (2 * h), s))
    for (d1, s1), (d2, s2) in zip(vals, vals[1:]):
        if abs(d1 - d2) <= 1e-5 * max(abs(d1), abs(d2)):
            return d1, s1
    return vals[-2]


def test_gpu_adjoint_against_central_differences(gpu):
    """32 seeded parameters: the 6 uniform E0/B0, 6 node E and 6 node B
    components, 14 initial velocity components -- each drawn among those
    whose gradient is at least 1 % of the largest of its kind (a component
    far below that is a cancellation of much larger terms, where FP32
    rounding of those terms decides the relative error).  The FP64 CPU
    adjoint's value is printed beside each."""
    c = case(n=(16, 16, 16), ppc=(2, 2), seed=23, b0=(0.05, -0.1, 0.2), vth_scale=2.0, tile=(8, 8, 8))
    c.b_modes, c.b_amp = 4, 2e-3
    cfg, eb, p, tp = build(c)
    K = 16
    lo, hi = (4, 4, 4), (12, 12, 12)
    with Emses(cfg) as g:
        g.upload_particles(p, tp)
        g.upload_field("eb", eb)
        g.fx_load()
        g.fx_store()
        p32, tp32 = g.download_particles()
        g.fx_load()
        o = O.Oracle(cfg, p32, tp32, eb)
        en, bn, e0b0 = node_fields(cfg, o)
        loss, gE, gB, g0, gv = g.fx_adjoint(K, 2, 4, 4, lo, hi, int(tp32.sum()))
    _, gE_o, gB_o, g0_o, gv_o = O.adjoint(cfg, K, 2, en, bn, e0b0, p32, lo, hi)

    def L(en_=en, bn_=bn, e0_=e0b0, p_=p32):
        return O.adjoint(cfg, K, 2, en_, bn_, e0_, p_, lo, hi, grad=False)[0]

    rng = np.random.default_rng(7)
    rows = []
    for k in range(6):
        def f(x, k=k):
            e = e0b0.copy()
            e[k] = x
            return L(e0_=e)
        scale = max(abs(e0b0[k]), np.abs(e0b0[:3] if k < 3 else e0b0[3:]).max())
        rows.append(("e0b0", k, g0[k], g0_o[k]) + fd_derivative(f, e0b0[k], scale))
    for arr, grad, go, name in ((en, gE, gE_o, "E"), (bn, gB, gB_o, "B")):
        big = np.argwhere(np.abs(go) >= 1e-2 * np.abs(go).max())
        for nd, comp in big[rng.choice(len(big), 6, replace=False)]:
            nd, comp = int(nd), int(comp)

            def f(x, nd=nd, comp=comp, arr=arr, name=name):
                a = arr.copy()
                a[nd, comp] = x
                return L(en_=a) if name == "E" else L(bn_=a)
            rows.append((name, nd * 3 + comp, grad[nd, comp], go[nd, comp]) +
                        fd_derivative(f, arr[nd, comp], np.abs(arr).max()))
    big = np.argwhere(np.abs(gv_o) >= 1e-2 * np.abs(gv_o).max())
    for m, comp in big[rng.choice(len(big), 14, replace=False)]:
        m, comp = int(m), int(comp)
        fld = ("vx", "vy", "vz")[comp]

        def f(x, m=m, fld=fld):
            q = p32.copy()
            q[fld][m] = x
            return L(p_=q)
        rows.append(("v", m * 3 + comp, gv[m, comp], gv_o[m, comp]) +
                    fd_derivative(f, p32[fld][m], np.abs(p32[fld]).max()))
    assert len(rows) == 32
    worst = 0.0
    for name, idx, gpu, cpu, fd, step in rows:
        err = abs(gpu - fd) / abs(fd)
        worst = max(worst, err)
        print(f"{name:5s} {idx:7d}  gpu {gpu: .9e}  fd {fd: .9e}  step {step:.0e}  rel {err:.1e}  "
              f"(FP64 adjoint {cpu: .9e}, rel {abs(cpu - fd) / abs(fd):.1e})")
        assert err <= 1e-4, (name, idx, gpu, fd, step)
    print("worst", worst)


def test_gpu_adjoint_on_the_16cube_copy_of_the_adjoint_workload(gpu):
    """The adjoint workload's plasma (32 ppc per species) on 16^3, K = 256
    steps with a checkpoint every 16 and a re-sort every 4, probe 8^3 at the
    centre: the GPU adjoint against the FP64 CPU adjoint (also checkpointed
    every 16 steps).  Over 256 steps the FP32 and FP64 trajectories part by
    rounding (and a particle that ends next to a face may take the other
    cell on one side), so the bound is 1e-3 relative L2 per gradient."""
    from ctca_b200 import inputs
    case4 = inputs.workload_case(4, scale=0.25)
    assert case4.n == (16, 16, 16) and case4.species[0].ppc == 32
    cfg = inputs.make_config(case4)
    eb = inputs.make_fields(case4)
    p, tp = inputs.make_particles(case4)
    lo, hi = (4, 4, 4), (12, 12, 12)
    with Emses(cfg) as g:
        g.upload_particles(p, tp)
        g.upload_field("eb", eb)
        g.fx_load()
        g.fx_store()
        p32, tp32 = g.download_particles()
        g.fx_load()
        o = O.Oracle(cfg, p32, tp32, eb)
        en, bn, e0b0 = node_fields(cfg, o)
        loss, gE, gB, g0, gv = g.fx_adjoint(256, 2, 16, 4, lo, hi, int(tp32.sum()))
    loss_o, gE_o, gB_o, g0_o, gv_o = O.adjoint(cfg, 256, 2, en, bn, e0b0, p32, lo, hi, ckpt=16)
    errs = {"loss": abs(loss - loss_o) / loss_o, "g0": rel_l2(g0, g0_o), "gE": rel_l2(gE, gE_o),
            "gB": rel_l2(gB, gB_o), "gv": rel_l2(gv, gv_o)}
    print("K=256 on 16^3 x 32 ppc:", errs)
    assert errs["loss"] < 1e-4
    for k in ("g0", "gE", "gB", "gv"):
        assert errs[k] < 1e-3, k
