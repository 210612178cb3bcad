"""Ensembles of independent EMSES particle runs on one GPU.

The reference runs one job per plasma: an ensemble of parameter draws is a
queue of separate runs.  Here many runs share the GPU at once: every run
keeps its own context (device buffers and stream) in the FP32 / fixed-point
form, and one CUDA graph (emsesg_batch_create) holds a block of steps of all
of them -- push, zigzag current and CIC charge, folds, and the tile sort
every S steps -- as independent branches, replayed until the runs have
taken their steps.  Small runs (16^3 cells fill 16 CTAs) leave most of the
148 SMs idle on their own; side by side in one graph they fill the GPU, and
the CPU launches one graph instead of about fifteen kernels per step and
run.

The tile shape, the sort interval S and the push CTA's share of a tile
region (rows per CTA: with fewer, a small grid's tiles spread over more
SMs) of each grid-size class come from an autotuner that times the
candidates on a batch of copies of the class's first run: tile and sort
interval first, then the rows per CTA for the best of those (the CTA itself
is fixed at 768 threads by the 736-slot rows of the layout).  Runs that do
not fit in device memory together go in waves.

Runs are drawn as stated for the ensemble workload: cubic periodic grids of
side 16, 24, 32, 48 or 64, electrons and ions (mass ratio 100, equal
temperatures) with particles per cell uniform in [8, 64] per species,
vth_e uniform in [0.02, 0.1], |B0| uniform in [0, 0.3] along a random
direction, and E from 4 seeded Fourier modes of amplitude 1e-3.
"""
from __future__ import annotations

import json
import math
import time
from dataclasses import dataclass, replace
from pathlib import Path

import numpy as np

from . import inputs
from .emses import Batch, Emses

SIDES = (16, 24, 32, 48, 64)
TILES = (4, 8)
SORTS = (1, 2, 4, 8)
CHUNKS = (256, 48, 16)  # rows of a tile region per push CTA
USTEP = 2


def ensemble_cases(count: int = 512, seed: int = 1005, sides=SIDES) -> list[inputs.Case]:
    """`count` seeded run descriptions of the ensemble workload."""
    rng = np.random.default_rng(seed)
    out = []
    for r in range(count):
        n = int(rng.choice(sides))
        ppc_e, ppc_i = (int(x) for x in rng.integers(8, 65, size=2))
        vth_e = float(rng.uniform(0.02, 0.1))
        bmag = float(rng.uniform(0.0, 0.3))
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        out.append(inputs.Case(
            n=(n, n, n),
            species=[inputs.Species(ppc_e, -1.0, vth_e), inputs.Species(ppc_i, 1.0 / 100.0, vth_e / 10.0)],
            b0=tuple(float(x) for x in bmag * d), e_modes=4, e_amp=1e-3, kmax=4 * 2 * math.pi / n,
            seed=seed * 1000 + r))
    return out


def particles(case: inputs.Case) -> int:
    ncell = case.n[0] * case.n[1] * case.n[2]
    return sum(s.ppc for s in case.species) * ncell


def split_runs(cases: list[inputs.Case], world: int, rank: int) -> list[int]:
    """Indices of the runs rank `rank` of `world` takes: the runs go, largest
    first, to the rank with the fewest particles so far (ties to the lower
    rank), so that every rank gets about the same particle-steps; no run is
    split and no data moves between ranks."""
    load = [0] * world
    mine = []
    for i in sorted(range(len(cases)), key=lambda i: (-particles(cases[i]), i)):
        r = min(range(world), key=lambda q: (load[q], q))
        load[r] += particles(cases[i])
        if r == rank:
            mine.append(i)
    return sorted(mine)


def run_bytes(case: inputs.Case) -> int:
    """Device memory of one run (context + FP32 form + sort scratch), with margin."""
    g = (case.n[0] + 9) * (case.n[1] + 9) * (case.n[2] + 9)
    return int(particles(case) * 260 + g * 480 + (48 << 20))


def open_run(case: inputs.Case, tile: int, chunk_rows: int = CHUNKS[0]) -> Emses:
    """A loaded run: context, fields, device-seeded plasma, FP32 form."""
    case = replace(case, sort_tile=(tile, tile, tile))
    g = Emses(inputs.make_config(case))
    g.upload_field("eb", inputs.make_fields(case))
    g.load_plasma(inputs.plasma(case))
    g.fx_load()
    g.fx_chunk_rows(chunk_rows)
    return g


def block_steps(sorts) -> int:
    b = 1
    for s in sorts:
        b = b * (2 * s) // math.gcd(b, 2 * s)
    return b


def _events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _ext(stream_ptr: int):
    import torch
    return torch.cuda.ExternalStream(stream_ptr)


def run_batch(runs: list[Emses], sorts: list[int], steps: int, warm_blocks: int = 1, stats: dict | None = None) -> float:
    """Seconds of device time for `steps` steps of every run through one graph
    (after warm_blocks untimed replays).  Steps beyond whole blocks run on the
    runs' own streams inside the timed region."""
    import torch
    block = block_steps(sorts)
    with Batch(runs, USTEP, block, sorts) as b:
        if stats is not None:
            stats["kernels"] = stats.get("kernels", 0) + b.kernels * (steps // block)
        bs = _ext(b.stream)
        if warm_blocks:
            b.launch(warm_blocks)
        torch.cuda.synchronize()
        e0, e1 = _events()
        e0.record(bs)
        nrep = steps // block
        b.launch(nrep)
        rem = steps - nrep * block
        if rem:
            for g, s in zip(runs, sorts):
                g.fx_run(USTEP, rem, s, use_graph=False)
            for g in runs:
                ev = torch.cuda.Event()
                ev.record(_ext(g.stream))
                bs.wait_event(ev)
        e1.record(bs)
        e1.synchronize()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3


def run_each(runs: list[Emses], sorts: list[int], steps: int, use_graph: bool, warm: int = 0) -> float:
    """Seconds of device time for the runs one after the other, each with
    its own launches (use_graph: its own per-run graph of 2*S steps)."""
    import torch
    total = 0.0
    for g, s in zip(runs, sorts):
        if warm:
            g.fx_run(USTEP, warm, s, use_graph=use_graph)
        st = _ext(g.stream)
        torch.cuda.synchronize()
        e0, e1 = _events()
        e0.record(st)
        g.fx_run(USTEP, steps, s, use_graph=use_graph)
        e1.record(st)
        e1.synchronize()
        total += e0.elapsed_time(e1) / 1e3
    return total


@dataclass
class Choice:
    tile: int
    sort_every: int
    ns_per_particle_step: float
    chunk_rows: int = CHUNKS[0]


class Autotuner:
    """Tile shape, sort interval and rows per push CTA per grid-size class
    (cubic side), timed on a batch of copies of the class's first run;
    results are kept in memory and, with `cache`, in a JSON file keyed by
    side."""

    def __init__(self, cache: str | Path | None = None, steps: int = 8, trial_particles: int = 32 << 20,
                 tiles=TILES, sorts=SORTS, chunks=CHUNKS):
        self.cache = Path(cache) if cache else None
        self.steps = steps
        self.trial_particles = trial_particles
        self.tiles = tiles
        self.sorts = sorts
        self.chunks = chunks
        self.table: dict[str, Choice] = {}
        self.trials: dict[str, list] = {}
        if self.cache and self.cache.exists():
            for k, v in json.loads(self.cache.read_text()).items():
                self.table[k] = Choice(**v)

    @staticmethod
    def key(case: inputs.Case) -> str:
        return f"side{case.n[0]}"

    def choose(self, case: inputs.Case) -> Choice:
        k = self.key(case)
        if k not in self.table:
            self.table[k] = self.tune(case)
            if self.cache:
                self.cache.write_text(json.dumps({a: vars(c) for a, c in self.table.items()}, indent=1))
        return self.table[k]

    def tune(self, case: inputs.Case) -> Choice:
        copies = int(min(16, max(1, self.trial_particles // max(particles(case), 1))))
        best = None
        trials = []
        for tile in self.tiles:
            if tile > min(case.n):
                continue
            runs = [open_run(replace(case, seed=case.seed + c), tile) for c in range(copies)]
            try:
                for s in self.sorts:
                    steps = max(self.steps, block_steps([s]))
                    t = run_batch(runs, [s] * copies, steps)
                    ns = t / (copies * particles(case) * steps) * 1e9
                    trials.append((tile, s, self.chunks[0], ns))
                    if best is None or ns < best.ns_per_particle_step:
                        best = Choice(tile, s, ns, self.chunks[0])
            finally:
                for g in runs:
                    g.close()
        # the rows per CTA, for the best tile and sort interval
        if best is not None and len(self.chunks) > 1:
            runs = [open_run(replace(case, seed=case.seed + c), best.tile) for c in range(copies)]
            try:
                steps = max(self.steps, block_steps([best.sort_every]))
                for rows in self.chunks[1:]:
                    for g in runs:
                        g.fx_chunk_rows(rows)
                    t = run_batch(runs, [best.sort_every] * copies, steps)
                    ns = t / (copies * particles(case) * steps) * 1e9
                    trials.append((best.tile, best.sort_every, rows, ns))
                    if ns < best.ns_per_particle_step:
                        best = Choice(best.tile, best.sort_every, ns, rows)
            finally:
                for g in runs:
                    g.close()
        self.trials[self.key(case)] = trials
        return best


def waves(cases: list[inputs.Case], budget: int) -> list[list[int]]:
    """Greedy packing of the runs (largest first) into waves that fit
    `budget` bytes of device memory."""
    order = sorted(range(len(cases)), key=lambda i: -run_bytes(cases[i]))
    out, cur, used = [], [], 0
    for i in order:
        b = run_bytes(cases[i])
        if cur and used + b > budget:
            out.append(cur)
            cur, used = [], 0
        cur.append(i)
        used += b
    if cur:
        out.append(cur)
    return out


def run_ensemble(cases: list[inputs.Case], steps: int, tuner: Autotuner, modes=("batch", "each"),
                 budget: int | None = None, warm: int = 4) -> dict:
    """Runs every case for `steps` steps in each of `modes` and returns the
    aggregate particle-steps per second of each:

      batch       one graph per wave holding all of its runs
      each        the runs one after the other, each with its own launches
      each_graph  the runs one after the other, each replaying its own graph
    """
    import torch
    if budget is None:
        free, _ = torch.cuda.mem_get_info()
        budget = int(free * 0.7)
    choice = [tuner.choose(c) for c in cases]
    secs = {m: 0.0 for m in modes}
    plan = waves(cases, budget)
    stats = {"kernels": 0}
    e2e = 0.0
    h2d = d2h = 0
    for w in plan:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        runs = [open_run(cases[i], choice[i].tile, choice[i].chunk_rows) for i in w]
        sorts = [choice[i].sort_every for i in w]
        torch.cuda.synchronize()
        e2e += time.perf_counter() - t0
        h2d += sum(g.field_size("eb") * 8 for g in runs)
        try:
            for m in modes:
                if m == "batch":
                    secs[m] += run_batch(runs, sorts, steps, warm_blocks=max(1, -(-warm // block_steps(sorts))),
                                         stats=stats)
                    t0 = time.perf_counter()
                    for g in runs:
                        g.download_field("rho")
                        g.download_field("aj")
                    e2e += time.perf_counter() - t0
                    d2h += sum((g.field_size("rho") + g.field_size("aj")) * 8 for g in runs)
                elif m == "each":
                    secs[m] += run_each(runs, sorts, steps, use_graph=False, warm=warm)
                elif m == "each_graph":
                    secs[m] += run_each(runs, sorts, steps, use_graph=True, warm=max(warm, 8))
                else:
                    raise ValueError(m)
            for g in runs:
                g.synchronize()
        finally:
            for g in runs:
                g.close()
    total = sum(particles(c) for c in cases) * steps
    if "batch" in secs:
        e2e += secs["batch"]  # device time of the batches; setup and downloads are wall time
    return {
        "e2e_seconds": e2e if "batch" in secs else None, "h2d_bytes": h2d, "d2h_bytes": d2h,
        "batch_kernels": stats["kernels"],
        "runs": len(cases), "steps": steps, "particles": sum(particles(c) for c in cases),
        "particle_steps": total, "waves": len(plan),
        "seconds": secs, "particle_steps_per_s": {m: total / t for m, t in secs.items() if t > 0},
        "choices": {k: vars(v) for k, v in tuner.table.items()},
    }
