"""Parity on the benchmark configurations, with the error of every quantity.

* The 32^3 case exactly (2 species x 16 ppc, 1,048,576 particles, mass ratio
  100, B0 = (0,0,0.2), E0 + 4 modes, 10 steps):
  - the plain FP64 drop-in (psolve1 + add_boundary_current, charge +
    add_boundary_charge) is bit-exact to the oracle in every particle record
    after every step, rho and J within 1e-12 (FP64 atomics order);
  - the FP32 form, started from its FP32-rounded state, against the oracle
    run on the FP32 form's own state every step (cells exact except next to
    a face, rho / J <= 1e-5 relative L2) and against the oracle running
    freely for the 10 steps (rho / J <= 1e-5).
* The physics of the 128^3 headline workload (mass ratio 1836, ion drift
  0.01 x, 8 E and 8 dB modes, sort every 4) on a 32^3 x 64 ppc grid
  (4,194,304 particles), the oracle re-seeded from the FP32 state every
  step: cells, sort counts and the sort permutation exact (particles next to
  a face reported), rho / J <= 1e-5, the FP64 kinetic energy and the
  continuity residual of the FP32 state checked.
Tolerances: rho / J 1e-5 relative L2 (the FP32 form's stated bound) on the
nodes 0..n (the guard layers of a periodic fold depend on which side of a
periodic face a particle is stored; see oracle.compare.nodes).  The 3-D
zigzag current is discontinuous where an end point crosses a face, so J is
compared with the oracle's current moved to the cells the FP32 form took
for the particles that FP32 rounding put on the other side of a face (each
listed; compare.j_error_corrected); the error before that move is printed.
Positions within 1e-6 cell; velocities within 1e-5 relative."""
import numpy as np
import pytest

from ctca_b200 import inputs
from ctca_b200.emses import FX_ROW_SLOTS, Emses
from oracle import compare as C
from oracle import oracle as O

from helpers import same_particles

pytestmark = pytest.mark.gpu

RHOJ_TOL = 1e-5
POS_TOL = 1e-6
VEL_TOL = 1e-5
FP64_TOL = 1e-12


def oracle_step(o, ustep=2):
    o.grdcrt()
    o.f["aj"][...] = 0.0
    o.psolve1(ustep, 0)
    o.reduce_aj()
    o.charge(0)
    o.reduce_rho("rho")


def config(case):
    cfg = inputs.make_config(case)
    eb = inputs.make_fields(case)
    p, tp = inputs.make_particles(case)
    return cfg, eb, p, tp


def test_config_32cube_fp64_dropin_ten_steps_bit_exact(gpu):
    case = inputs.workload_case(1)
    cfg, eb, p, tp = config(case)
    assert int(tp.sum()) == 1048576
    with Emses(cfg) as g:
        g.upload_particles(p, tp)
        g.upload_field("eb", eb)
        o = O.Oracle(cfg, p, tp, eb)
        for step in range(10):
            g.grdcrt(1)
            g.zero_field("aj")
            g.psolve1(1, 2, 0)
            g.reduce_aj()
            g.charge(1, 0)
            g.reduce_rho("rho")
            oracle_step(o)
            pg, tpg = g.download_particles()
            assert np.array_equal(tpg, o.totalp)
            assert same_particles(pg, o.pbuf), f"step {step}"
            assert C.rel_l2(g.download_field("aj"), o.f["aj"]) < FP64_TOL
            assert C.rel_l2(g.download_field("rho"), o.f["rho"]) < FP64_TOL
        assert C.rel_l2(g.energy(), o.energy()) < FP64_TOL


def fx_start(cfg, eb, p, tp):
    """A context with the FP32 form loaded and its FP32-rounded state as
    FP64 records (the common start of both sides)."""
    g = Emses(cfg)
    g.upload_particles(p, tp)
    g.upload_field("eb", eb)
    g.fx_load()
    g.fx_store()
    p32, tp32 = g.download_particles()
    g.fx_load()
    return g, p32, tp32


def check_step(cfg, g, o, start, label):
    """The FP32 form's state and fields after a step against the oracle's
    (same start): returns the error report, asserting the bounds."""
    g.fx_store()
    pg, tpg = g.download_particles()
    rep = C.particle_errors(cfg, pg, o.pbuf)
    jg = g.download_field("aj")
    rep["rho"] = C.field_errors(g.download_field("rho"), o.f["rho"], cfg)
    rep["aj"] = C.field_errors(jg, o.f["aj"], cfg)
    raw, same = C.j_error_corrected(cfg, jg, o.f["aj"], start, pg, o.pbuf, rep["mismatched"])
    rep["aj"]["l2_rel_same_cells"] = same
    print(label, {k: v for k, v in rep.items() if k != "mismatched"})
    assert np.array_equal(tpg, o.totalp)
    assert rep["alive_mismatch"] == 0
    assert rep["cell_mismatch_off_band"] == 0, label
    assert rep["pos_max_abs"] < POS_TOL, label
    assert rep["vel_max_rel"] < VEL_TOL, label
    assert rep["rho"]["l2_rel"] < RHOJ_TOL, label
    assert same < RHOJ_TOL, label
    return rep, pg


def test_config_32cube_fp32_form_ten_steps(gpu):
    case = inputs.workload_case(1)
    case.sort_tile = (8, 8, 8)
    cfg, eb, p, tp = config(case)
    g, p32, tp32 = fx_start(cfg, eb, p, tp)
    free = O.Oracle(cfg, p32, tp32, eb)  # runs the 10 steps on its own
    cur = p32
    for step in range(10):
        o = O.Oracle(cfg, cur, tp32, eb)  # re-seeded from the FP32 state
        oracle_step(o)
        free_start = free.pbuf.copy()
        oracle_step(free)
        g.fx_step(2, False)
        _, after = check_step(cfg, g, o, cur, f"32^3 step {step}")
        # the free-running oracle: its cells differ from the FP32 form's only
        # next to faces, and J by the zigzag jumps of those particles
        rf = C.particle_errors(cfg, after, free.pbuf)
        assert rf["cell_mismatch_off_band"] == 0
        assert C.field_errors(g.download_field("rho"), free.f["rho"], cfg)["l2_rel"] < RHOJ_TOL
        raw, same = C.j_error_corrected(cfg, g.download_field("aj"), free.f["aj"], free_start, after, free.pbuf,
                                        rf["mismatched"])
        print(f"free-running step {step}: J {raw:.2e} ({same:.2e} with the FP32 form's cells), cells differing "
              f"{rf['cell_mismatch']}")
        assert same < RHOJ_TOL
        cur = after
    g.close()


def test_config_headline_physics_32cube_64ppc(gpu):
    """The headline workload's physics on 32^3 x 64 ppc, 8 steps with a
    re-sort after steps 4 and 8; the oracle starts every step from the FP32
    form's state."""
    case = inputs.workload_case(2, scale=0.25)
    assert case.n == (32, 32, 32) and case.species[0].ppc == 64
    cfg, eb, p, tp = config(case)
    g, p32, tp32 = fx_start(cfg, eb, p, tp)
    tile = case.sort_tile
    cur, tp_cur = p32, tp32      # the state a step starts from
    last_sorted = p32            # the records right after the last sort
    rho_old = None
    for step in range(8):
        o = O.Oracle(cfg, cur, tp_cur, eb)
        o.charge(0)
        o.reduce_rho("rho")
        rho_o_old = o.f["rho"].copy()
        oracle_step(o)
        g.fx_step(2, False)
        rep, after = check_step(cfg, g, o, cur, f"headline physics step {step}")
        # FP64 checks on the FP32 state: the kinetic energy of the FP32 form's
        # own particles, and against the oracle's FP64 particles
        eg = g.fx_energy()
        assert C.rel_l2(eg, O.Oracle(cfg, after, tp_cur, eb).energy()) < FP64_TOL
        assert C.rel_l2(eg, o.energy()) < VEL_TOL
        res, rmax = g.fx_continuity()
        rho_new, aj = g.download_field("rho"), g.download_field("aj")
        res_o = C.continuity_residual(cfg, rho_o_old, o.f["rho"], o.f["aj"])
        print(f"continuity residual {res:.3e} (oracle {res_o:.3e}), max |rho| {rmax:.3e}")
        if rho_old is None:
            assert np.isnan(res)
        else:
            assert res == C.continuity_residual(cfg, rho_old, rho_new, aj)
            assert res < 1e-3 * rmax and res_o < 1e-3 * rmax
        rho_old = rho_new
        if step % 4 == 3:
            # the re-sort: per-cell counts and the permutation, exact
            g.fx_sort()
            g.fx_store()
            srt, tps = g.download_particles()
            b0 = np.concatenate([[0], np.cumsum(tp_cur)])
            b1 = np.concatenate([[0], np.cumsum(tps)])
            assert np.array_equal(tps, [(after[b0[s]:b0[s + 1]]["nid"] != -1).sum() for s in range(cfg.nspec)])
            assert np.array_equal(C.cell_histogram(cfg, srt), C.cell_histogram(cfg, after))
            if rep["cell_mismatch"] == 0:
                assert np.array_equal(C.cell_histogram(cfg, srt), C.cell_histogram(cfg, o.pbuf))
            for s in range(cfg.nspec):
                before, moved = last_sorted[b0[s]:b0[s + 1]], after[b0[s]:b0[s + 1]]
                exp = C.sort_order(cfg, tile, FX_ROW_SLOTS, before, moved)
                assert same_particles(srt[b1[s]:b1[s + 1]], moved[exp]), f"species {s} permutation"
                if rep["cell_mismatch"] == 0:
                    okeys = C.tile_key(cfg, tile, o.pbuf[b0[s]:b0[s + 1]])[0]
                    assert np.array_equal(C.sort_order(cfg, tile, FX_ROW_SLOTS, before, moved, keys=okeys), exp)
            cur, tp_cur, last_sorted = srt, tps, srt
        else:
            cur = after
    g.close()


def test_fx_energy_fp32_only_matches(gpu):
    """emsesg_fx_energy on an FP32-only context (no FP64 records) equals the
    same state's energy in a context with records, bit for bit."""
    case = inputs.workload_case(2, scale=0.125)
    case.species[0].ppc = case.species[1].ppc = 8
    cfg = inputs.make_config(case)
    eb = inputs.make_fields(case)
    pl = inputs.plasma(case)
    out = []
    for flags in (0, 1):
        cfg.flags = flags
        with Emses(cfg) as g:
            g.upload_field("eb", eb)
            if flags:
                g.fx_load_plasma(pl)
            else:
                g.load_plasma(pl)
                g.fx_load()
            for s in range(3):
                g.fx_step(2, s == 1)
            out.append(g.fx_energy())
            if not flags:
                g.fx_store()
                pg, tpg = g.download_particles()
                o = O.Oracle(cfg, pg, tpg, eb)
                assert C.rel_l2(out[-1], o.energy()) < FP64_TOL
    assert np.array_equal(out[0], out[1])
