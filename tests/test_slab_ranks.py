"""The exchange of the z-slab decomposition (ctca_b200.slabs.exchange_step)
on gloo processes (CPU), with a toy slab in place of the GPU context: the
protocol -- counts, then particle records, then the z border planes, each
round's sends and receives posted together, arrivals from below before
those from above -- on 2 and 3 ranks reproduces one slab holding the whole
periodic grid.

The toy slab keeps the interfaces of ContextIO with the same plane ranges
(rho: one plane each way, from 0 / to n+1 and from n / to -1; J: three,
from -1..1 / to n+2..n+4 and from n-1..n+1 / to -4..-2) and the same folds:
particles on a periodic line move by their velocity; every particle adds
its "current" at the cell it moves into (unwrapped: a guard cell when it
leaves), a particle that stays adds its "charge" to the two nodes around
it, one that leaves goes to the outbox (in the neighbour's frame) and its
charge is added by the receiver."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from ctca_b200 import slabs

RECW = slabs.REC_BYTES // 8  # float64 words of a record


class ToySlab:
    def __init__(self, z, v, nz):
        self.z = np.asarray(z, dtype=np.float64).copy()
        self.v = np.asarray(v, dtype=np.float64).copy()
        self.n = nz
        self.device = torch.device("cpu")
        self.rho = np.zeros(nz + 3, dtype=np.int64)  # nodes -1..n+1
        self.j = np.zeros(nz + 9, dtype=np.int64)    # nodes -4..n+4
        self.out = [np.zeros((0, RECW)), np.zeros((0, RECW))]

    def _charge(self, z):
        k = np.floor(z).astype(np.int64)
        np.add.at(self.rho, k + 1, 3)   # node k
        np.add.at(self.rho, k + 2, 5)   # node k + 1

    def begin(self, ustep):
        self.rho[:] = 0
        self.j[:] = 0
        a = self.z + self.v * ustep
        k = np.floor(a).astype(np.int64)
        np.add.at(self.j, k + 4, 7)
        stay = (k >= 0) & (k < self.n)
        self._charge(a[stay])
        out = []
        for d, m in ((0, k < 0), (1, k >= self.n)):
            r = np.zeros((int(m.sum()), RECW))
            r[:, 0] = a[m] + (self.n if d == 0 else -self.n)
            r[:, 1] = self.v[m]
            out.append(r)
        self.out = out
        self.z, self.v = a[stay], self.v[stay]
        return np.array([[self.out[0].shape[0], self.out[1].shape[0]]], dtype=np.int64)

    def outbox(self, spec, d, n):
        return torch.from_numpy(self.out[d].ravel().view(np.uint8))

    def new_records(self, n):
        return torch.empty(n * slabs.REC_BYTES, dtype=torch.uint8)

    def arrive(self, spec, buf, n):
        r = buf.numpy().view(np.float64).reshape(n, RECW)
        self._charge(r[:, 0])
        self.z = np.concatenate([self.z, r[:, 0]])
        self.v = np.concatenate([self.v, r[:, 1]])

    def border(self):
        pass

    def planes(self, which):
        n = self.n
        rk = {0: 0, 1: n, 2: -1, 3: n + 1}[which]
        jk = {0: -1, 1: n - 1, 2: -4, 3: n + 2}[which]
        return (torch.from_numpy(self.rho[rk + 1:rk + 2]), torch.from_numpy(self.j[jk + 4:jk + 7]))

    def fold(self):
        n = self.n
        self.rho[1] += self.rho[0]          # node 0 += node -1
        self.rho[n + 1] += self.rho[n + 2]  # node n += node n + 1
        self.j[3:6] += self.j[0:3]          # nodes -1..1 += -4..-2
        self.j[n + 3:n + 6] += self.j[n + 6:n + 9]

    def end(self, do_sort):
        self.fold()

    def wait(self):
        pass


def whole_run(z, v, nz, steps):
    """One toy slab holding the whole periodic line (its own neighbour)."""
    t = ToySlab(z, v, nz)
    for _ in range(steps):
        t.begin(1)
        for d in (1, 0):
            r = t.out[d]
            t.arrive(1, torch.from_numpy(r.ravel().view(np.uint8).copy()), r.shape[0])
        for src, dst in ((1, 2), (0, 3)):
            a, b = t.planes(src)
            c, e = t.planes(dst)
            c.copy_(a.clone())
            e.copy_(b.clone())
        t.fold()
    return t


def line(nz, seed=3, n=400):
    rng = np.random.default_rng(seed)
    # under a cell a step, as in the push (which deposits a particle's
    # current no further than one guard cell out)
    return rng.uniform(0, nz, n), rng.uniform(-0.95, 0.95, n)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, nz, steps, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        z, v = line(nz)
        nzl = nz // world
        m = (np.floor(z) >= rank * nzl) & (np.floor(z) < (rank + 1) * nzl)
        t = ToySlab(z[m] - rank * nzl, v[m], nzl)
        moved = 0
        for _ in range(steps):
            moved += int(slabs.exchange_step(t, dist, None, rank, world, 1, False).sum())
        # the global counters: one all-reduce over the ranks
        tot = slabs.reduce_counts(np.array([[t.z.size, moved]]), dist)
        q.put((rank, t.rho[1:nzl + 2].copy(), t.j[4:nzl + 5].copy(), np.sort(t.z + rank * nzl), moved, tot))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_slab_exchange_over_gloo_ranks(world):
    nz, steps = 12 * world, 5
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, nz, steps, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ref = whole_run(*line(nz), nz, steps)
    nzl = nz // world
    rho = np.zeros(nz + 1, dtype=np.int64)
    j = np.zeros(nz + 1, dtype=np.int64)
    moved_all = sum(o[4] for o in out)
    for r, rr, jr, zr, moved, tot in out:
        assert moved > 0
        assert tot.shape == (1, 2) and tot[0, 0] == ref.z.size and tot[0, 1] == moved_all
        rho[r * nzl:(r + 1) * nzl + 1] = rr
        j[r * nzl:(r + 1) * nzl + 1] = jr
        # the shared node of two slabs holds the same value on both
        if r > 0:
            assert rr[0] == prev_rho_top and jr[0] == prev_j_top
        prev_rho_top, prev_j_top = rr[-1], jr[-1]
    assert np.array_equal(rho, ref.rho[1:nz + 2])
    assert np.array_equal(j, ref.j[4:nz + 5])
    # positions: the slabs move in their own frames (shifted by whole cells),
    # so they agree to the rounding of the shift
    zs = np.sort(np.concatenate([o[3] for o in out]))
    assert zs.size == ref.z.size and np.max(np.abs(zs - np.sort(ref.z))) < 1e-12
