"""Benchmark of the EMSES particle hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: 128^3 periodic cells, electrons + ions x 64 particles per cell
(268,435,456 particles), mass ratio 1836, ion drift 0.01 x, B0 = (0,0,0.1)
plus 8 seeded dB modes and 8 seeded E modes of amplitude 1e-3, dt = 0.5,
cell sort every 4 steps (seeded synthetic inputs in the reference's internal
units, ctca_b200/inputs.py).  One step = field relocation (grdcrt), push,
zigzag current and CIC charge into int64 fixed point, guard folding, FP64
rho / J outputs, plus the sort + compaction on every 4th step.

`value` is particle-steps per second of the FP32 / fixed-point form with the
state resident in HBM (7.5 GB of particles, well above the 126 MB L2, so no
L2 flush is needed).  `e2e` is the same metric through the C ABI with host
buffers: every step uploads eb from pinned host memory and downloads rho and
J.  `fp64_dropin` reports the plain FP64 drop-in (64-byte records) on the
same workload.  With --gpus N every rank runs its own replica (the path has
no data exchange on one rank: weak scaling, replicas only).

--cells N [--ppc P] shrinks the grid (and particles per cell) for profiler
captures; the headline line is the default 128^3 x 64 workload.

Four more workloads ride on the headline line (skip them with --no-extras):
`adjoint` times the reverse mode through K = 256 steps of a 64^3 periodic
grid with 32 particles per cell per species (checkpoints every 16 steps,
loss = sum of Jx^2 over an 8^3 probe) against the same K forward steps;
`ensemble` runs a bounded sample of the ensemble workload (independent runs
of side 16..64 in one CUDA graph) against the same runs launched one after
the other; `em_loop` and `es_loop` are 12 steps of the --workload em and es
loops below on the headline grid.  --workload ensemble prints the full
ensemble line instead (512 runs x 200 steps by default).

--workload em and --workload es run the headline plasma self-consistently
with the field solve on the device every step: the EM leapfrog (bfield,
push, bfield, efield, border exchange) or the electrostatic loop (push, rho,
FFT Poisson solve, E from phi).

--workload slabs runs the headline plasma on a grid cut into z slabs
(ctca_b200/slabs.py): with torchrun and N GPUs one 128^3 slab per GPU
(128 x 128 x 128N cells, weak scaling) exchanging the particles that change
slab and the border planes of rho and J over NCCL every step; on one GPU two
slabs of half the grid in one process against the grid as one context.

--impl reference times the reference's CPU path (the oracle restatement of
psolve1 + charge; the Fortran reference cannot be built here) on the host
cores, on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "push+deposit particles/s & % HBM roofline: FP32-fixedpt vs FP64 plain; adj/fwd"
UNIT = "particle-steps/s"
SORT_EVERY = 4
# Algorithmic bytes of one particle-step (FP32 form, S = 4, 128 particles
# per cell): 2*28 (push read+write) + (2*28+8)/4 (sort) + (24+32)/128 (grid).
B_ALG_STEP = 2 * 28 + (2 * 28 + 8) / SORT_EVERY + (24 + 32) / 128
B_ALG_PUSH = 2 * 28  # the fused push + deposit kernel, per particle
# The plain FP64 drop-in (64-byte records): push read + write 128, charge read
# 64, sort (128 + 8)/S, grid (48 + 32)/128.
B_ALG_FP64 = 2 * 64 + 64 + (2 * 64 + 8) / SORT_EVERY + (48 + 32) / 128


def peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling (every 50 ms) during the timed region (read only):
    the sampler is running before the region starts, and only the samples
    taken inside it are summarised."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []  # (host time, fields)
        self.proc = None
        self.t0 = self.t1 = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
            deadline = time.time() + 3.0
            while not self.samples and time.time() < deadline:
                time.sleep(0.01)
        except Exception:
            self.proc = None
        self.t0 = time.time()
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append((time.time(), [x.strip() for x in line.split(",")]))

    def __exit__(self, *exc):
        self.t1 = time.time()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.reader.join(timeout=2)

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        inside = [f for t, f in self.samples if self.t0 is not None and self.t0 <= t <= (self.t1 or t)]
        for s in inside or [f for _, f in self.samples[-1:]]:
            try:
                sm.append(float(s[1]))
                mx = float(s[2])
                for n, v in zip(names, s[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("gloo", timeout=timedelta(seconds=600))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world, x: float) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# --------------------------------------------------------------- CPU baseline
def headline_case(cells: int = 0, ppc: int = 0):
    """The headline workload (128^3, 2 species x 64 ppc, mass ratio 1836,
    ion drift, 8 E and 8 dB modes), or a smaller copy for profiler captures."""
    from ctca_b200 import inputs
    case = inputs.workload_case(2)
    if cells:
        case.n = (cells, cells, cells)
        case.kmax = 4 * 2 * math.pi / cells
        for sp in case.species:
            sp.ppc = ppc or sp.ppc
    return case


def headline_config(case, npart: int, world: int) -> dict:
    return {"workload": f"{case.n[0]}^3 periodic, 2 species x {case.species[0].ppc} ppc ({npart:,} particles), "
                        "mass ratio 1836, sort every 4; FP32 cell+offset particles, int64 rho/J at 2^40",
            "l2": f"inputs larger than L2 ({npart * 28 / 1e9:.2f} GB particle state)",
            "parallelism": f"replicas x{world}"}


def cpu_blocks(case, layers: int | None, threads: int, seconds: float, min_steps: int, max_steps: int,
               restore: bool = True, warmup: int = 1) -> dict:
    """Times the oracle's psolve1 + charge in the reference's one rank per
    core (oracle.Blocks) on the first `layers` z layers of `case` (all of it
    when None): particle-steps per second over the timed steps, after
    `warmup` untimed ones (with `restore`)."""
    from ctca_b200 import inputs
    from oracle import oracle as O
    cfg = inputs.make_config(case)
    eb = inputs.make_fields(case)
    cells = None if layers is None else case.n[0] * case.n[1] * layers
    p, tp = inputs.make_particles(case, cells=cells)
    o = O.Oracle(cfg, p[:0], [0] * cfg.nspec, eb)
    o.grdcrt()
    b = O.Blocks(cfg, o.f["wrk"], p, tp, threads)
    del p, o
    for _ in range(warmup if restore else 0):
        b.step(2)  # untimed
    ts = []
    while len(ts) < max_steps and (len(ts) < min_steps or sum(ts) < seconds):
        ts.append(b.step(2, restore))
    out = {"value": b.particles * len(ts) / sum(ts), "threads": b.threads, "particles": b.particles,
           "steps": len(ts), "s_per_step": sum(ts) / len(ts)}
    b.close()
    return out


def cpu_baseline(threads: int) -> dict:
    """The reference's CPU path, timed on the host cores: the headline
    workload's plasma (a sample of its z layers at the full 64 ppc) on one
    thread and on all threads, and the 32^3 x 16 ppc case for 10 steps."""
    from ctca_b200 import inputs
    allt = cpu_blocks(headline_case(), 8, threads, 3.0, 3, 20)
    one = cpu_blocks(headline_case(), 1, 1, 2.0, 2, 10)
    c1 = inputs.workload_case(1)
    c1_one = cpu_blocks(c1, None, 1, 0.0, 10, 10, restore=False)
    c1_all = cpu_blocks(c1, None, threads, 0.0, 10, 10, restore=False)
    return {
        "value": allt["value"], "unit": UNIT, "cores": allt["threads"], "kind": "port",
        "sample": (f"first 8 z layers of the 128^3 x 2 species x 64 ppc workload ({allt['particles']:,} particles, "
                   "the same plasma drawn on the host), the oracle's psolve1 + charge (FP64, g++ -O3), one block "
                   f"of x rows per thread as one rank per core, {allt['steps']} steps each from the same particles"),
        "single_thread": {"value": one["value"], "unit": UNIT, "cores": 1,
                          "sample": f"first z layer ({one['particles']:,} particles), {one['steps']} steps"},
        "config_32cube_16ppc": {"workload": "32^3 periodic, 2 species x 16 ppc (1,048,576 particles), mass ratio "
                                            "100, B0 (0,0,0.2), E0 + 4 modes, 10 steps",
                                "threads_1": c1_one["value"], "threads_all": c1_all["value"],
                                "cores": c1_all["threads"], "unit": UNIT},
    }


def run_reference(args, world, rank):
    """The reference's CPU path on the host cores (rank 0 only): the oracle's
    psolve1 + charge, one block of x rows per thread, on the first 8 z layers
    of the headline workload at its full 64 ppc; every timed step is one step
    of that sample from the same particles."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    case = headline_case()
    total = sum(sp.ppc for sp in case.species) * case.n[0] * case.n[1] * case.n[2]
    r = cpu_blocks(case, 8, threads, 0.0, args.steps, args.steps, warmup=max(args.warmup, 0))
    sample = (f"first 8 z layers of the workload ({r['particles']:,} particles, the same plasma drawn on the host), "
              "the oracle's psolve1 + charge (FP64 restatement of the reference; the Fortran reference is not "
              "buildable: no Fortran/MPI/HDF5/FFTW toolchain), one block of x rows per thread as one rank per core; "
              "each step from the same particles")
    line = {
        "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": r["steps"],
        "warmup": args.warmup, "ms_per_step": r["s_per_step"] * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": headline_config(case, total, 1),
        "sample": sample,
        "cpu_baseline": {"value": r["value"], "unit": UNIT, "cores": r["threads"], "kind": "port", "sample": sample},
        "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def fx_fp64_checks(g) -> dict:
    """The FP64 checks of the FP32 state after the last step: kinetic energy
    per species and component (energy.F90), and the continuity residual
    max |rho_new - rho_old + 2 div J| of the last step with max |rho|."""
    e = g.fx_energy()
    res, rmax = g.fx_continuity()
    return {"kinetic_energy": [[float(x) for x in row] for row in e], "continuity_residual": res,
            "max_rho": rmax, "note": "FP64 over the FP32 state of the last timed step"}


# --------------------------------------------------------------- accuracy (checker)
def accuracy_report(steps: int = 4) -> dict:
    """Errors of the FP32 form against the FP64 oracle on the headline
    workload's physics at 32^3 x 64 ppc (4,194,304 particles), the oracle
    started every step from the FP32 form's own state, with the re-sort after
    the 4th step: worst case over the steps of every quantity."""
    from ctca_b200 import inputs
    from ctca_b200.emses import FX_ROW_SLOTS, Emses
    from oracle import compare as C
    from oracle import oracle as O

    case = inputs.workload_case(2, scale=0.25)
    cfg = inputs.make_config(case)
    eb = inputs.make_fields(case)
    p, tp = inputs.make_particles(case)
    worst = {"pos_max_abs": 0.0, "pos_rms": 0.0, "vel_max_rel": 0.0, "vel_l2_rel": 0.0, "rho_l2_rel": 0.0,
             "rho_max_rel": 0.0, "j_l2_rel": 0.0, "j_max_rel": 0.0, "j_l2_rel_same_cells": 0.0, "cell_mismatch": 0, "cell_mismatch_off_band": 0,
             "near_face": 0, "alive_mismatch": 0, "sort_count_mismatch_cells": 0, "permutation_mismatch": 0,
             "energy_rel": 0.0, "energy_fp64_reproducible": True, "continuity_residual": 0.0,
             "continuity_residual_oracle": 0.0, "continuity_max_rho": 0.0}
    with Emses(cfg) as g:
        g.upload_particles(p, tp)
        g.upload_field("eb", eb)
        g.fx_load()
        g.fx_store()
        cur, tpc = g.download_particles()
        g.fx_load()
        last_sorted = cur
        for step in range(steps):
            o = O.Oracle(cfg, cur, tpc, eb)
            o.charge(0)
            o.reduce_rho("rho")
            rho_o_old = o.f["rho"].copy()
            o.grdcrt()
            o.f["aj"][...] = 0.0
            o.psolve1(2, 0)
            o.reduce_aj()
            o.charge(0)
            o.reduce_rho("rho")
            g.fx_step(2, False)
            g.fx_store()
            after, _ = g.download_particles()
            rep = C.particle_errors(cfg, after, o.pbuf)
            for k in ("pos_max_abs", "pos_rms", "vel_max_rel", "vel_l2_rel"):
                worst[k] = max(worst[k], rep[k])
            for k in ("cell_mismatch", "cell_mismatch_off_band", "near_face", "alive_mismatch"):
                worst[k] += rep[k]
            for name, key in (("rho", "rho"), ("aj", "j")):
                fe = C.field_errors(g.download_field(name), o.f[name], cfg)
                worst[key + "_l2_rel"] = max(worst[key + "_l2_rel"], fe["l2_rel"])
                worst[key + "_max_rel"] = max(worst[key + "_max_rel"], fe["max_rel"])
            _, same = C.j_error_corrected(cfg, g.download_field("aj"), o.f["aj"], cur, after, o.pbuf,
                                          rep["mismatched"])
            worst["j_l2_rel_same_cells"] = max(worst["j_l2_rel_same_cells"], same)
            eg = g.fx_energy()
            worst["energy_rel"] = max(worst["energy_rel"], C.rel_l2(eg, o.energy()))
            worst["energy_fp64_reproducible"] &= bool(np.array_equal(eg, g.fx_energy()))
            res, rmax = g.fx_continuity()
            if not math.isnan(res):
                worst["continuity_residual"] = max(worst["continuity_residual"], res)
                worst["continuity_max_rho"] = max(worst["continuity_max_rho"], rmax)
                worst["continuity_residual_oracle"] = max(
                    worst["continuity_residual_oracle"],
                    C.continuity_residual(cfg, rho_o_old, o.f["rho"], o.f["aj"]))
            if step % SORT_EVERY == SORT_EVERY - 1:
                g.fx_sort()
                g.fx_store()
                srt, tps = g.download_particles()
                worst["sort_count_mismatch_cells"] += int(np.sum(C.cell_histogram(cfg, srt)
                                                                 != C.cell_histogram(cfg, o.pbuf)))
                b0 = np.concatenate([[0], np.cumsum(tpc)])
                b1 = np.concatenate([[0], np.cumsum(tps)])
                for sp in range(cfg.nspec):
                    before, moved = last_sorted[b0[sp]:b0[sp + 1]], after[b0[sp]:b0[sp + 1]]
                    okeys = C.tile_key(cfg, case.sort_tile, o.pbuf[b0[sp]:b0[sp + 1]])[0]
                    exp = C.sort_order(cfg, case.sort_tile, FX_ROW_SLOTS, before, moved, keys=okeys)
                    got = srt[b1[sp]:b1[sp + 1]]
                    if got.size != exp.size:
                        worst["permutation_mismatch"] += abs(got.size - exp.size)
                        continue
                    same = np.all(np.stack([got[f] == moved[exp][f] for f in ("x", "y", "z", "vx", "vy", "vz")]), 0)
                    worst["permutation_mismatch"] += int((~same).sum())
                cur, tpc, last_sorted = srt, tps, srt
            else:
                cur = after
    worst["workload"] = (f"the headline physics (mass ratio 1836, ion drift, 8 E and 8 dB modes) on 32^3 x 64 ppc "
                         f"({int(tp.sum()):,} particles), {steps} steps with the re-sort after step {SORT_EVERY}; the "
                         "FP64 oracle started every step from the FP32 form's state; worst step (max) or total over "
                         "the steps (counts)")
    worst["definitions"] = ("pos in cells, vel relative to the largest |v|, rho/J relative L2 and max on the "
                            "nodes 0..n (j_l2_rel_same_cells: with the oracle's zigzag current moved to the "
                            "cells the FP32 form took for the particles FP32 rounding put across a face); cell "
                            "mismatches counted, those farther than 4 FP32 ulps from every face must be 0; "
                            "permutation against the tile sort's definition with the oracle's cells; energy = FP64 "
                            "kinetic energy of the FP32 state vs the oracle's; continuity = max |rho_new - rho_old + "
                            "2 div J| in FP64 (the 3-D zigzag's cubic remainder)")
    return worst


# --------------------------------------------------------------- GPU arm
def time_adjoint(K: int = 256, ckpt: int = 16, sort_every: int = SORT_EVERY) -> dict:
    """Forward K steps vs the reverse mode through them (emsesg_fx_adjoint)
    on the 64^3 x 32 ppc adjoint workload."""
    import torch
    from ctca_b200 import inputs
    from ctca_b200.emses import Emses
    case = inputs.workload_case(4)
    cfg = inputs.make_config(case)
    eb = inputs.make_fields(case)
    lo = tuple(case.n[d] // 2 - 4 for d in range(3))
    hi = tuple(x + 8 for x in lo)
    with Emses(cfg) as g:
        g.upload_field("eb", eb)
        g.load_plasma(inputs.plasma(case))
        g.fx_load()
        npart = int(g.fx_counts().sum())
        st = torch.cuda.ExternalStream(g.stream)
        g.fx_run(2, 2 * sort_every, sort_every, use_graph=False)  # warm-up
        g.synchronize()
        g.load_plasma(inputs.plasma(case))
        g.fx_load()
        g.synchronize()
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record(st)
        g.fx_run(2, K, sort_every, use_graph=False)
        e1.record(st)
        e1.synchronize()
        # warm-up call: allocates the adjoint workspace (kept between calls);
        # the velocity gradients go to pinned host memory
        gv_pinned = torch.empty((npart, 3), dtype=torch.float64, pin_memory=True)
        g.load_plasma(inputs.plasma(case))
        g.fx_load()
        g.fx_adjoint(K, 2, ckpt, sort_every, lo, hi, npart, gv_out=gv_pinned.numpy())
        g.load_plasma(inputs.plasma(case))
        g.fx_load()
        g.synchronize()
        e1b = torch.cuda.Event(enable_timing=True)
        e1b.record(st)
        loss, gE, gB, g0, gv = g.fx_adjoint(K, 2, ckpt, sort_every, lo, hi, npart, gv_out=gv_pinned.numpy())
        e2.record(st)
        e2.synchronize()
        fwd = e0.elapsed_time(e1) / 1e3
        adj = e1b.elapsed_time(e2) / 1e3
    return {"workload": f"{case.n[0]}^3 periodic, 2 species x 32 ppc ({npart:,} particles), K={K}, "
                        f"checkpoint every {ckpt}, sort every {sort_every}, loss = sum Jx^2 over an 8^3 probe",
            "forward_s": fwd, "adjoint_call_s": adj,
            "reverse_over_forward": (adj - fwd) / fwd, "call_over_forward": adj / fwd,
            "note": "the adjoint call runs the forward (with checkpoints, keeping the probe Jx of every "
                    "step) and then the reverse sweep, which recomputes each checkpoint segment with move-only "
                    "steps; reverse_over_forward = (call - forward) / forward; second call (the first allocates "
                    "the workspace); includes the copy of the gradients to host (pinned memory)",
            "loss": loss}


def ensemble_sample(runs: int, steps: int) -> dict:
    from ctca_b200 import ensemble
    cases = ensemble.ensemble_cases(runs)
    tuner = ensemble.Autotuner()
    out = ensemble.run_ensemble(cases, steps, tuner, modes=("batch", "each"))
    v = out["particle_steps_per_s"]
    out["batch_over_each"] = v["batch"] / v["each"]
    out["workload"] = (f"first {runs} of the 512 seeded ensemble runs (cubic periodic, side 16..64, "
                       f"ppc U[8,64] per species, mass ratio 100), {steps} steps each")
    return out


def run_ours(args, world, rank, local):
    import torch
    from ctca_b200 import inputs
    from ctca_b200.emses import Emses, select_device

    torch.cuda.set_device(local)
    select_device(local)
    # args.cells: a smaller copy of the workload for profiler captures (not the headline)
    case = headline_case(args.cells, args.ppc)
    cfg = inputs.make_config(case)
    eb = inputs.make_fields(case)
    npart = sum(cfg.capacity[i] for i in range(cfg.nspec))
    g = Emses(cfg)
    g.load_plasma(inputs.plasma(case, seed=case.seed + 1000 * rank))
    g.upload_field("eb", eb)
    stream = torch.cuda.ExternalStream(g.stream)

    def timed(fn, steps):
        barrier(world)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for s in range(steps):
            fn(s)
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        barrier(world)
        return max_over_ranks(world, e0.elapsed_time(e1) / 1e3)

    # ---- plain FP64 drop-in (64-byte records): grdcrt, psolve1, folds, charge, sort every 4
    def fp64_step(s):
        g.grdcrt(1)
        g.zero_field("aj")
        g.psolve1(1, 2, 0)
        g.reduce_aj()
        if s % SORT_EVERY == SORT_EVERY - 1:
            g.spsort(1)
        g.charge(1, 0)
        g.reduce_rho("rho")

    k64 = max(1, min(args.steps, args.fp64_steps))
    for s in range(args.warmup):
        fp64_step(s)
    g.synchronize()
    t64 = timed(fp64_step, k64)
    g.synchronize()

    # ---- FP32 / fixed-point form
    g.fx_load()
    step_i = [0]

    def fx_step(s):
        g.fx_step(2, (step_i[0] % SORT_EVERY) == SORT_EVERY - 1)
        step_i[0] += 1

    for s in range(args.warmup):
        fx_step(s)
    g.set_profiling(True)
    g.profile_reset()
    with Clocks(local) as clk:
        t = timed(fx_step, args.steps)
    prof = g.profile()
    g.set_profiling(False)
    fp64_checks = fx_fp64_checks(g)

    # ---- end to end through the C ABI with host buffers
    eb_host = torch.empty(eb.size, dtype=torch.float64, pin_memory=True)
    eb_host.numpy()[:] = eb.reshape(-1)
    nr = g.field_size("rho")
    na = g.field_size("aj")
    rho_host = torch.empty(nr, dtype=torch.float64, pin_memory=True)
    aj_host = torch.empty(na, dtype=torch.float64, pin_memory=True)
    lib = g.lib

    # per step: this step's eb up (copied beside the previous step's sort,
    # after its rho / J reached the host), the step, rho and J down (beside
    # this step's sort); the host has rho and J before it uploads the next eb
    def e2e_step(s):
        lib.emsesg_upload_field_async(g.h, 0, eb_host.data_ptr())
        rc = lib.emsesg_fx_step_download(g.h, 2, 1 if (step_i[0] % SORT_EVERY) == SORT_EVERY - 1 else 0,
                                         rho_host.data_ptr(), aj_host.data_ptr())
        step_i[0] += 1
        if rc:
            raise RuntimeError(f"emsesg_fx_step_download: {rc}")

    ke2e = max(1, min(args.steps, args.e2e_steps))
    te2e = timed(e2e_step, ke2e)
    g.synchronize()

    value = world * npart * args.steps / t
    hbm, peak_kind = peaks()
    ms, launches = prof.get("fx_push", (0.0, 0))
    avg_launch_s = ms / 1e3 / max(launches, 1)
    parts_per_launch = npart  # one launch pushes every species (grid.y = species)
    achieved = B_ALG_PUSH * parts_per_launch / avg_launch_s / 1e9 if launches else None
    traffic = None
    tfile = ROOT / "profiles" / "traffic.json"
    if tfile.exists():
        tb = json.loads(tfile.read_text()).get("fx_push_bytes_per_particle")
        if tb:
            traffic = tb * parts_per_launch
    step_time = t / args.steps
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_time * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+i64", "data": "synthetic",
        "config": headline_config(case, npart, world),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": (achieved / hbm) if achieved else None, "traffic": traffic,
                     "kernel": "fx_push", "peak_kind": peak_kind,
                     "bytes_per_particle_alg": B_ALG_PUSH,
                     "step_frac": B_ALG_STEP * npart / step_time / 1e9 / hbm},
        "e2e": {"value": world * npart * ke2e / te2e, "unit": UNIT,
                "h2d_bytes_per_step": int(eb.size * 8), "d2h_bytes_per_step": int((nr + na) * 8)},
        "fp64_dropin": {"value": world * npart * k64 / t64, "unit": UNIT, "steps": k64,
                        "ms_per_step": t64 / k64 * 1e3,
                        "fp32_over_fp64": (value / (world * npart * k64 / t64)),
                        "bytes_per_particle_step_alg": B_ALG_FP64,
                        "roofline_frac": B_ALG_FP64 * npart / (t64 / k64) / 1e9 / hbm},
        "fp64_checks": fp64_checks,
        "gpu_launches": int(sum(n for _, n in prof.values())),
        "kernels_ms": {k: round(v[0], 3) for k, v in sorted(prof.items(), key=lambda kv: -kv[1][0])},
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_extras and not args.cells:
        out["adjoint"] = time_adjoint()
        out["ensemble"] = ensemble_sample(args.ensemble_runs, args.ensemble_steps)
        out["em_loop"] = loop_section(local, es=False)
        out["es_loop"] = loop_section(local, es=True)
    if rank == 0 and world == 1 and not args.no_cpu:
        out["cpu_baseline"] = cpu_baseline(os.cpu_count() or 1)
        out["accuracy"] = accuracy_report()
    g.close()
    if rank == 0:
        print(json.dumps(out), flush=True)


def run_slabs_line(args, world, rank, local):
    """The headline plasma on a grid cut into z slabs (ctca_b200/slabs.py):
    with N GPUs one 128^3 slab per GPU, a grid of 128 x 128 x 128N (weak
    scaling), the particles that change slab and the z border planes of rho
    and J exchanged every step over NCCL (device to device); on one GPU two
    slabs of 128 x 128 x 64 in one process, against the same grid as one
    context (what the decomposition itself costs).  Each slab draws its
    plasma on its device (its own seed)."""
    import torch
    from ctca_b200 import inputs, slabs
    from ctca_b200.emses import Emses, select_device
    torch.cuda.set_device(local)
    select_device(local)
    case = headline_case(args.cells, args.ppc)
    nslab = max(world, 2)
    nzs = case.n[2] if world > 1 else case.n[2] // 2
    gcase = headline_case(args.cells, args.ppc)
    gcase.n = (case.n[0], case.n[1], nzs * nslab)
    cfg = inputs.make_config(gcase)
    eb = inputs.make_fields(gcase)
    sub = slabs.slab_config(cfg, nslab)
    ppc = sum(s.ppc for s in case.species)
    outbox = max(1 << 16, case.n[0] * case.n[1] * ppc // 4)
    steps, warm = args.steps, max(3, args.warmup)

    def slab_plasma(r):
        scase = headline_case(args.cells, args.ppc)
        scase.n = (case.n[0], case.n[1], nzs)
        return inputs.plasma(scase, seed=case.seed + 7919 * (r + 1))

    if world == 1:
        grp = slabs.SlabGroup(cfg, eb, None, None, nslab, outbox, plasmas=[slab_plasma(r) for r in range(nslab)])
        npart = int(grp.counts().sum())
        for s in range(warm):
            grp.step(2, s % SORT_EVERY == SORT_EVERY - 1)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for s in range(steps):
            grp.step(2, (warm + s) % SORT_EVERY == SORT_EVERY - 1)
        torch.cuda.synchronize()
        e1.record()
        e1.synchronize()
        t = e0.elapsed_time(e1) / 1e3
        moved = grp.migrated
        grp.close()
        # the same grid as one context
        w = Emses(cfg)
        w.load_plasma(inputs.plasma(gcase, seed=case.seed + 7919))
        w.upload_field("eb", eb)
        w.fx_load()
        for s in range(warm):
            w.fx_step(2, s % SORT_EVERY == SORT_EVERY - 1)
        st = torch.cuda.ExternalStream(w.stream)
        w.synchronize()
        e0.record(st)
        for s in range(steps):
            w.fx_step(2, (warm + s) % SORT_EVERY == SORT_EVERY - 1)
        e1.record(st)
        e1.synchronize()
        tw = e0.elapsed_time(e1) / 1e3
        nw = int(w.fx_counts().sum())
        w.close()
        value = npart * steps / t
        line = {"metric": "slab decomposition particle-steps/s", "value": value, "unit": UNIT, "n_gpus": 1,
                "steps": steps, "warmup": warm, "ms_per_step": t / steps * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32+i64", "data": "synthetic",
                "config": {"workload": f"{gcase.n[0]}x{gcase.n[1]}x{gcase.n[2]} periodic cut into {nslab} z "
                                       f"slabs on one GPU, 2 species x {case.species[0].ppc} ppc "
                                       f"({npart:,} particles), sort every 4",
                           "parallelism": f"{nslab} slabs, one process"},
                "whole_grid": {"value": nw * steps / tw, "ms_per_step": tw / steps * 1e3},
                "decomposed_over_whole": (value / (nw * steps / tw)),
                "changed_slab_per_step": (moved / (steps + warm))}
        print(json.dumps(line), flush=True)
        return
    import torch.distributed as dist
    nccl = dist.new_group(backend="nccl")
    g = Emses(sub)
    g.load_plasma(slab_plasma(rank))
    g.upload_field("eb", slabs.slab_field(cfg, eb, "eb", rank, nslab))
    g.fx_load()
    g.fx_slab(True, outbox)
    io = slabs.ContextIO(g)
    n_local = int(g.fx_counts().sum())
    for s in range(warm):
        slabs.exchange_step(io, dist, nccl, rank, world, 2, s % SORT_EVERY == SORT_EVERY - 1)
    st = torch.cuda.ExternalStream(g.stream)
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    moved = 0
    for s in range(steps):
        moved += int(slabs.exchange_step(io, dist, nccl, rank, world, 2,
                                         (warm + s) % SORT_EVERY == SORT_EVERY - 1).sum())
    e1.record(st)
    e1.synchronize()
    torch.cuda.synchronize()
    barrier(world)
    t = max_over_ranks(world, e0.elapsed_time(e1) / 1e3)
    cnt = torch.tensor([float(n_local), float(moved)], dtype=torch.float64)
    dist.all_reduce(cnt)
    g.close()
    dist.destroy_process_group(nccl)
    if rank == 0:
        npart, moved_all = int(cnt[0].item()), int(cnt[1].item())
        print(json.dumps({"metric": "slab decomposition particle-steps/s", "value": npart * steps / t, "unit": UNIT,
                          "n_gpus": world, "steps": steps, "warmup": warm, "ms_per_step": t / steps * 1e3,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+i64",
                          "data": "synthetic",
                          "config": {"workload": f"{gcase.n[0]}x{gcase.n[1]}x{gcase.n[2]} periodic, one "
                                                 f"{case.n[0]}x{case.n[1]}x{nzs} z slab per GPU, 2 species x "
                                                 f"{case.species[0].ppc} ppc ({npart:,} particles), sort every 4",
                                     "parallelism": f"z slabs x{world}, NCCL point-to-point"},
                          "changed_slab_per_step": moved_all / steps}), flush=True)


def run_ensemble_line(args, world, rank, local):
    """The ensemble workload: runs split across ranks by particle count
    (ensemble.split_runs), each rank's runs in one graph per wave; value =
    all runs' particle-steps over the slowest rank's device time."""
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no ensemble runner: each "
                              "run is a separate job of the CPU path, timed by --impl reference"}), flush=True)
        return
    import torch
    from ctca_b200 import ensemble
    from ctca_b200.emses import select_device
    torch.cuda.set_device(local)
    select_device(local)
    cases = ensemble.ensemble_cases(args.ensemble_runs)
    mine = [cases[i] for i in ensemble.split_runs(cases, world, rank)]
    tuner = ensemble.Autotuner()
    with Clocks(local) as clk:
        out = ensemble.run_ensemble(mine, args.ensemble_steps, tuner, modes=("batch", "each"))
    t_batch = max_over_ranks(world, out["seconds"]["batch"])
    t_each = max_over_ranks(world, out["seconds"]["each"])
    total = sum(ensemble.particles(c) for c in cases) * args.ensemble_steps
    line = {
        "metric": METRIC, "value": total / t_batch, "unit": UNIT, "n_gpus": world, "steps": args.ensemble_steps,
        "warmup": 4, "ms_per_step": t_batch / args.ensemble_steps * 1e3, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32+i64", "data": "synthetic",
        "config": {"workload": f"ensemble of {len(cases)} independent periodic runs (side 16..64, ppc U[8,64] per "
                               f"species, mass ratio 100), {args.ensemble_steps} steps each, one CUDA graph per "
                               "wave of runs that fit in memory",
                   "l2": "runs larger than L2 together (GBs of particle state per wave)",
                   "parallelism": f"runs split over {world} GPU(s)"},
        "one_launch_per_run": {"value": total / t_each, "unit": UNIT, "seconds": t_each},
        "batch_over_each": t_each / t_batch,
        "autotuner": out["choices"], "waves": out["waves"],
        "e2e": {"value": total / out["e2e_seconds"], "unit": UNIT, "note": "setup + batch + rho/J download, wall",
                "h2d_bytes_per_step": int(out["h2d_bytes"] / args.ensemble_steps),
                "d2h_bytes_per_step": int(out["d2h_bytes"] / args.ensemble_steps)},
        "gpu_launches": max_over_ranks(world, out["batch_kernels"]),
        "clocks": clk.summary(),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


BODY_NPR = 4096  # entries of each velocity table of the body workload


_BODY_TABLES = {}


def body_tables(case) -> dict:
    """The velocity tables of the body workload, built by the reference's
    own table code (ctca_b200/tables.py) from one random stream seeded with
    the case's seed: per species the open-boundary tables (flux through the
    z faces of the drifting Maxwellian, Maxwellian x / y), then the emission
    tables of the photoelectrons (flux and tangential Maxwellian of
    vth = 0.01)."""
    key = (case.seed, tuple((s.vth, s.drift[2]) for s in case.species))
    if key not in _BODY_TABLES:
        from ctca_b200 import inputs, tables
        renv = inputs.units()["renv"]
        rng = tables.Ranu0(case.seed)
        out = {"species": []}
        for s in case.species:
            t = tables.inflow_tables(BODY_NPR, 1, (0.0, 0.0, s.drift[2] * renv), s.vth * renv, s.vth * renv, rng)
            out["species"].append({"vzf": t["vzf"], "vzb": t["vzb"], "vxr": t["vxr"], "vyr": t["vyr"]})
        em = tables.emission_tables(BODY_NPR, BODY_NPR, 0.0, 0.01 * renv, 0.01 * renv, 0.0, rng)
        out["vn"], out["vt"] = em["vnormf"], em["vtangf"]
        _BODY_TABLES[key] = out
    return _BODY_TABLES[key]


def body_plan(case, scale: float) -> dict:
    """Per-step injection of the body workload drawn on the device: tables
    and counts (the rates of body_injection)."""
    nx, ny, nz = case.n
    tb = body_tables(case)
    plan = {"nemit": int(round((1 << 20) * scale ** 3)), "vn": tb["vn"], "vt": tb["vt"], "inflow": []}
    counts = [0, 0]
    for isp, s in enumerate(case.species):
        vd = s.drift[2]
        st = tb["species"][isp]
        for front, sgn in ((True, +1.0), (False, -1.0)):
            n = int(round(s.ppc * nx * ny * _flux(vd, s.vth, sgn) * case.dt))
            if n:
                plan["inflow"].append((isp + 1, front, n, st["vzf"] if front else st["vzb"], st["vxr"], st["vyr"]))
                counts[isp] += n
    counts[0] += 2 * plan["nemit"]
    plan["counts"] = counts
    return plan


def body_inject_device(g, case, plan, seed: int, step: int):
    """One step's injection of the body workload with the device supervisors."""
    body = case.bodies[0]
    for q, (spec, front, n, vz, vx, vy) in enumerate(plan["inflow"]):
        g.fx_inflow_z(spec, front, n, vz, vx, vy, 2.0, seed, 10 + q, step * n)
    if plan["nemit"]:
        g.fx_emit(1, 1, body["xupc"], (body["ylpc"], body["yupc"]), (body["zlpc"], body["zupc"]), plan["nemit"],
                  plan["vn"], plan["vt"], seed, 1, step * plan["nemit"])


def _flux(mu, sig, sign):
    """E[(sign v)+] for v ~ N(mu, sig^2)."""
    from math import erf, exp, pi, sqrt
    m = sign * mu
    return sig * exp(-0.5 * (m / sig) ** 2) / sqrt(2 * pi) + m * 0.5 * (1 + erf(m / sig / sqrt(2)))


def _body_step(job):
    """The injected records of one step of the body workload (see
    body_injection); runs in a worker process."""
    case, scale, seed, step = job
    from ctca_b200 import inject
    nx, ny, nz = case.n
    rng = np.random.default_rng([seed, step])
    body = case.bodies[0]
    nemit = int(round((1 << 20) * scale ** 3))
    tb = body_tables(case)
    recs = []
    for isp, s in enumerate(case.species):
        vd = s.drift[2]
        st = tb["species"][isp]
        parts = []
        for front, sgn in ((True, +1.0), (False, -1.0)):
            cnt = s.ppc * nx * ny * _flux(vd, s.vth, sgn) * case.dt
            n = int(cnt) + (1 if rng.random() < cnt - int(cnt) else 0)
            if n:
                parts.append(inject.inflow_z(front, n, nx, ny, nz, st["vzf"] if front else st["vzb"], st["vxr"],
                                             st["vyr"], 2.0, rng, spec=isp + 1))
        if isp == 0 and nemit:
            parts.append(inject.emit_rectangle(1, body["xupc"], (body["ylpc"], body["yupc"]),
                                               (body["zlpc"], body["zupc"]), nemit, tb["vn"], tb["vt"], rng, spec=1))
        recs.append(np.concatenate(parts))
    return recs


def body_injection(case, steps: int, scale: float, seed: int):
    """Records injected before each step of the body workload: inflow of
    both species through the z faces at the rate of their drifting
    Maxwellian flux (particles per step = ppc * face cells * flux * dt), and
    2^20 (x scale^3) photoelectrons from the body's +x face with vth = 0.01
    (pairs of an anti-particle on the face and a particle just off it).
    Drawn in worker processes (started before any CUDA call).  Returns
    [step][species] record arrays."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor
    jobs = [(case, scale, seed, k) for k in range(steps)]
    workers = max(1, min(len(jobs), (os.cpu_count() or 2) - 1, 32))
    with ProcessPoolExecutor(workers, mp_context=mp.get_context("spawn")) as ex:
        return list(ex.map(_body_step, jobs))


def run_body_line(args, world, rank, local):
    """The body workload: 256x256x512 cells, open z, solar-wind electrons and
    ions (24 ppc each, 1.61e9 particles) drifting along -z past a 32x32x16
    conducting box that absorbs them (int64 counts per surface cell) and
    emits 2^20 photoelectrons a step from its +x face, inflow through the z
    faces; B0 = (0.05, 0, 0.1), E = 0.  An FP32-only context (no FP64
    particle buffer) holds it on one GPU.  Each timed step injects the
    step's records -- drawn on the device (emsesg_fx_emit,
    emsesg_fx_inflow_z), or with --host-inject drawn on the host and
    uploaded from pinned memory -- and pushes; sort every 4 steps."""
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the body workload (1.6e9 particles) is timed on "
                              "the GPU only; the reference CPU path is timed by the default workload"}), flush=True)
        return
    import torch
    from ctca_b200 import inputs
    from ctca_b200.emses import Emses, select_device
    torch.cuda.set_device(local)
    select_device(local)
    scale = args.body_scale
    case = inputs.workload_case(3, scale)
    steps, warm = args.steps, args.warmup
    nstep_all = warm + steps + 5
    seed = case.seed + 17 * rank
    if args.host_inject:
        inj = body_injection(case, nstep_all, scale, seed=seed)
        counts = [[int(r.size) for r in st] for st in inj]
        # the step's records come from pinned host memory (asynchronous uploads)
        pinned = [[torch.from_numpy(r.view(np.uint8)).pin_memory() for r in st] for st in inj]
    else:
        plan = body_plan(case, scale)
        counts = [plan["counts"]] * nstep_all
    add = [sum(st[i] for st in counts) for i in range(2)]
    ncell = case.n[0] * case.n[1] * case.n[2]
    cap = [int(s.ppc * ncell * 1.01) + add[i] + (1 << 20) for i, s in enumerate(case.species)]
    cfg = inputs.make_config(case, capacity=cap)
    cfg.flags = 1  # EMSESG_FLAG_FP32_ONLY
    g = Emses(cfg)
    g.fx_load_plasma(inputs.plasma(case, seed=case.seed + 1000 * rank))
    stream = torch.cuda.ExternalStream(g.stream)
    k = [0]

    def step():
        if args.host_inject:
            recs = inj[k[0]]
            for isp in range(2):
                if recs[isp].size:
                    g.fx_inject_raw(isp + 1, pinned[k[0]][isp].data_ptr(), recs[isp].size)
        else:
            body_inject_device(g, case, plan, seed, k[0])
        g.fx_step(2, k[0] % SORT_EVERY == SORT_EVERY - 1)
        k[0] += 1

    for _ in range(warm):
        step()
    g.synchronize()
    n0 = int(g.fx_counts().sum())
    g.set_profiling(True)
    g.profile_reset()
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        e0.record(stream)
        for _ in range(steps):
            step()
        e1.record(stream)
        e1.synchronize()
    torch.cuda.synchronize()
    barrier(world)
    t = max_over_ranks(world, e0.elapsed_time(e1) / 1e3)
    prof = g.profile()
    g.set_profiling(False)
    n1 = int(g.fx_counts().sum())
    body_checks = fx_fp64_checks(g)
    g.fx_background(False)  # add_background_charge from the surface counts
    body_checks["background_charge_total"] = float(g.download_field("rhobk").sum())
    inj_bytes = (sum(int(r.nbytes) for st in inj[warm:warm + steps] for r in st) if args.host_inject
                 else 0)
    # end to end: the same steps plus rho and J to host after each one
    nr, na = g.field_size("rho"), g.field_size("aj")
    rho_h = torch.empty(nr, dtype=torch.float64, pin_memory=True)
    aj_h = torch.empty(na, dtype=torch.float64, pin_memory=True)
    ke = min(5, nstep_all - k[0])
    ne0 = int(g.fx_counts().sum())
    g.synchronize()
    t0 = time.perf_counter()
    for _ in range(ke):
        step()
        g.lib.emsesg_download_field(g.h, 4, rho_h.data_ptr())
        g.lib.emsesg_download_field(g.h, 2, aj_h.data_ptr())
    g.synchronize()
    te = time.perf_counter() - t0
    ne1 = int(g.fx_counts().sum())
    surf = g.fx_surface()
    counters = g.get_counters().as_dict()
    hbm, peak_kind = peaks()
    ms, launches = prof.get("fx_push", (0.0, 0))
    npart = 0.5 * (n0 + n1)
    achieved = B_ALG_PUSH * npart / (ms / 1e3 / launches) / 1e9 if launches else None
    out = {
        "metric": METRIC, "value": world * npart * steps / t, "unit": UNIT, "n_gpus": world, "steps": steps,
        "warmup": warm, "ms_per_step": t / steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+i64", "data": "synthetic",
        "config": {"workload": f"{case.n[0]}x{case.n[1]}x{case.n[2]} cells, open z, 2 species x 24 ppc "
                               f"({n0:,} particles at the start), drift -0.08 z, box body "
                               f"{int(case.bodies[0]['xupc'] - case.bodies[0]['xlpc'])}x"
                               f"{int(case.bodies[0]['yupc'] - case.bodies[0]['ylpc'])}x"
                               f"{int(case.bodies[0]['zupc'] - case.bodies[0]['zlpc'])} absorbing with int64 "
                               f"surface counts, {counts[0][0]:,} electron and {counts[0][1]:,} ion records "
                               "injected a step (z inflow + photoemission pairs, drawn on the "
                               f"{'host' if args.host_inject else 'device'}), sort every 4, FP32-only context",
                   "l2": "inputs larger than L2", "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": (achieved / hbm) if achieved else None, "traffic": None, "kernel": "fx_push",
                     "peak_kind": peak_kind, "bytes_per_particle_alg": B_ALG_PUSH},
        "e2e": {"value": world * 0.5 * (ne0 + ne1) * ke / te, "unit": UNIT, "steps": ke,
                "h2d_bytes_per_step": int(inj_bytes / steps), "d2h_bytes_per_step": int((nr + na) * 8)},
        "particles": {"start": n0, "end": n1},
        "fp64_checks": body_checks,
        "absorbed": {"influx_e": int(counters["influx"][0].sum()), "influx_i": int(counters["influx"][1].sum()),
                     "surface_net_e": int(surf[0].sum()), "surface_net_i": int(surf[1].sum()),
                     "escaped_e": int(counters["nesc"][0]), "escaped_i": int(counters["nesc"][1])},
        "gpu_launches": int(sum(n for _, n in prof.values())),
        "kernels_ms": {kk: round(v[0], 3) for kk, v in sorted(prof.items(), key=lambda kv: -kv[1][0])},
        "clocks": clk.summary(),
    }
    g.close()
    if rank == 0:
        print(json.dumps(out), flush=True)


def run_em_line(args, world, rank, local, es=False):
    """The headline workload run self-consistently with the fields on the
    device: each step is bfield, push + J + rho, bfield, efield and the eb
    border exchange (emsesg_fx_em_step; tcs = 2 (c dt)^2 = 0.125 in internal
    units for c dt / dx = 0.5); sort every 4 steps.  With es (--workload es)
    the electrostatic loop instead: push + rho without the current
    (emsesg_fx_step_es, psolve2 + charge), then E from rho by the FFT
    Poisson solve (emsesg_esfield)."""
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the reference's field solver is not built (no "
                              "Fortran toolchain); its CPU particle path is timed by the default workload"}),
                  flush=True)
        return
    out = field_loop(args.cells, args.ppc, args.steps, args.warmup, world, rank, local, es)
    if rank == 0:
        print(json.dumps(out), flush=True)


def field_loop(cells, ppc, steps, warmup, world, rank, local, es):
    """One timed run of the EM (or, with es, the electrostatic) loop of
    run_em_line; returns its line."""
    import torch
    from ctca_b200 import inputs
    from ctca_b200.emses import Emses, select_device
    torch.cuda.set_device(local)
    select_device(local)
    case = headline_case(cells, ppc)
    cfg = inputs.make_config(case)
    g = Emses(cfg)
    g.upload_field("eb", inputs.make_fields(case))
    g.fx_load_plasma(inputs.plasma(case, seed=case.seed + 1000 * rank))
    npart = int(g.fx_counts().sum())
    stream = torch.cuda.ExternalStream(g.stream)
    k = [0]

    def step():
        if es:
            g.fx_step_es(2, k[0] % SORT_EVERY == SORT_EVERY - 1)
            g.esfield(1, check=False)
        else:
            g.fx_em_step(2, k[0] % SORT_EVERY == SORT_EVERY - 1, 0.125)
        k[0] += 1

    for _ in range(warmup):
        step()
    g.synchronize()
    g.set_profiling(True)
    g.profile_reset()
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        e0.record(stream)
        for _ in range(steps):
            step()
        e1.record(stream)
        e1.synchronize()
    torch.cuda.synchronize()
    barrier(world)
    t = max_over_ranks(world, e0.elapsed_time(e1) / 1e3)
    prof = g.profile()
    fields = ("es_pack", "es_fft", "es_divide", "es_unpack", "es_efield") if es else ("bfield", "efield", "exchange_eb")
    field_ms = sum(prof.get(n, (0.0, 0))[0] for n in fields)
    out = {"metric": METRIC, "value": world * npart * steps / t, "unit": UNIT, "n_gpus": world,
           "steps": steps, "warmup": warmup, "ms_per_step": t / steps * 1e3,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+i64 (fields f64)",
           "data": "synthetic",
           "config": {"workload": f"{case.n[0]}^3 periodic, 2 species x {case.species[0].ppc} ppc ({npart:,} "
                                  "particles), " + ("electrostatic loop on the device each step (push and "
                                  "rho without the current, FFT Poisson solve, E from phi)" if es else "EM fields advanced on the "
                                  "device each step (bfield, push, bfield, efield, border exchange)") +
                                  ", sort every 4",
                      "l2": "inputs larger than L2", "parallelism": f"replicas x{world}"},
           "field_step_ms": field_ms / steps,
           "gpu_launches": int(sum(n for _, n in prof.values())),
           "kernels_ms": {kk: round(v[0], 3) for kk, v in sorted(prof.items(), key=lambda kv: -kv[1][0])},
           "clocks": clk.summary()}
    g.close()
    return out


def loop_section(local, es):
    """The EM / electrostatic loop on the headline grid for the default line
    (12 timed steps after 3 warm-up steps, three sorts)."""
    o = field_loop(0, 0, 12, 3, 1, 0, local, es)
    return {k: o[k] for k in ("value", "unit", "ms_per_step", "steps", "warmup", "field_step_ms", "config",
                              "gpu_launches", "clocks")}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--fp64-steps", type=int, default=8)
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cells", type=int, default=0, help="grid side of a smaller profiling case (default 128)")
    ap.add_argument("--ppc", type=int, default=0, help="particles per cell per species with --cells")
    ap.add_argument("--no-extras", action="store_true", help="skip the adjoint, ensemble and loop sections")
    ap.add_argument("--workload", default="particle_step",
                    choices=["particle_step", "ensemble", "body", "em", "es", "slabs"])
    ap.add_argument("--body-scale", type=float, default=1.0, help="grid scale of the body workload (1: 256x256x512)")
    ap.add_argument("--host-inject", action="store_true",
                    help="body workload: draw the injected records on the host (else on the device)")
    ap.add_argument("--ensemble-runs", type=int, default=None)
    ap.add_argument("--ensemble-steps", type=int, default=None)
    args = ap.parse_args()
    world, rank, local = dist_setup()
    try:
        if args.workload == "body":
            run_body_line(args, world, rank, local)
        elif args.workload in ("em", "es"):
            run_em_line(args, world, rank, local, es=args.workload == "es")
        elif args.workload == "slabs":
            run_slabs_line(args, world, rank, local)
        elif args.workload == "ensemble":
            args.ensemble_runs = args.ensemble_runs or 512
            args.ensemble_steps = args.ensemble_steps or 200
            run_ensemble_line(args, world, rank, local)
        elif args.impl == "reference":
            run_reference(args, world, rank)
        else:
            args.ensemble_runs = args.ensemble_runs or 64
            args.ensemble_steps = args.ensemble_steps or 40
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
