"""Domain decomposition of the FP32 form in z slabs.

The reference spreads a run over MPI ranks with OhHelp: every rank owns a
subdomain with its own field arrays (guards included), pushes the particles
in it, sends the particles that left to the neighbour that owns their new
position (oh2_transbound / exchange_particles,
lib/ohhelp/ohhelp-1.1.1/ohhelp2.c:103-123, 333-384) and exchanges the
border planes of rho and J before folding the guards
(oh3_exchange_borders, ohhelp3.c:959-1046; add_boundary_charge,
charge.F90:214-412; add_boundary_current, psolve1.F90:859-1079).

Here the grid, periodic in z, is cut into P slabs of equal thickness along
z, one per rank (one GPU each), and each slab is a context in slab mode
(emsesg_fx_slab).  A step of every slab is

  1. emsesg_fx_slab_begin: the push; the particles that leave through a z
     face go to an outbox per direction, in the neighbour's frame;
  2. the outbox records go to the two neighbours (ring: direction 1 up, 0
     down);
  3. emsesg_fx_slab_arrive: the particles from below, then from above, into
     the tail zone, their charge into rho;
  4. emsesg_fx_slab_border: the x / y border exchange of rho and J;
  5. the z border planes of the int64 rho and J accumulators go to the
     neighbours, into their guard planes;
  6. emsesg_fx_slab_end: the guard folds and the FP64 fields.

Only steps 2 and 5 cross ranks.  `SlabGroup` runs all slabs in one process (one
GPU or several, copies through the device), `SlabRank` one slab per process
with torch.distributed (NCCL between GPUs: the records and planes go device
to device, no host round trip).  On the nodes 0..nz of each slab the FP64
rho and J equal those of one context holding the whole grid up to the FP32
rounding of the push's run sums (both are sums of the same int64
contributions per particle; which particles share a run differs).
"""
from __future__ import annotations

import numpy as np

from .emses import PARTICLE_DTYPE, Config, Emses, field_extents, field_shape

REC_BYTES = PARTICLE_DTYPE.itemsize


def slab_config(cfg: Config, nslab: int, capacity_factor: float = 1.25) -> Config:
    """The configuration of one of nslab slabs of cfg's grid: nz / nslab
    cells along z (nz divisible by nslab), the species capacities scaled by
    1 / nslab times capacity_factor."""
    if cfg.nz % nslab:
        raise ValueError(f"nz = {cfg.nz} is not divisible by {nslab} slabs")
    c = type(cfg).from_buffer_copy(cfg)
    c.nz = cfg.nz // nslab
    for s in range(cfg.nspec):
        c.capacity[s] = int(np.ceil(cfg.capacity[s] / nslab * capacity_factor))
    return c


def slab_field(cfg: Config, a: np.ndarray, name: str, r: int, nslab: int) -> np.ndarray:
    """Slab r's copy of a node field of the whole grid (numpy (z, y, x, c)
    with the field's guards), its z planes taken periodically."""
    nc, lo, ex, ey, ez = field_extents(cfg, name)
    nzl = cfg.nz // nslab
    ezl = ez - cfg.nz + nzl
    k = (np.arange(ezl) + lo + r * nzl) % cfg.nz - lo
    return np.ascontiguousarray(a.reshape(ez, ey, ex, nc)[k])


def slab_particles(cfg: Config, p: np.ndarray, tp, r: int, nslab: int) -> tuple[np.ndarray, np.ndarray]:
    """The records of slab r (z in [r nz / nslab, (r + 1) nz / nslab)), z
    shifted into its frame, per species in order; and their counts."""
    nzl = cfg.nz // nslab
    z0 = r * nzl
    out, counts, b = [], [], 0
    for s in range(cfg.nspec):
        q = p[b:b + int(tp[s])]
        b += int(tp[s])
        m = (np.floor(q["z"]) >= z0) & (np.floor(q["z"]) < z0 + nzl)
        qs = q[m].copy()
        qs["z"] -= z0
        out.append(qs)
        counts.append(qs.size)
    return np.concatenate(out) if out else np.zeros(0, dtype=PARTICLE_DTYPE), np.array(counts, dtype=np.int64)


def assemble(cfg: Config, name: str, parts: list) -> np.ndarray:
    """The field of the whole grid on its nodes 0..n from the slabs' fields
    (each slab's nodes 0..nz / nslab; the shared plane from the slab that
    owns it as its node 0), numpy (nz + 1, ny + 1, nx + 1, c)."""
    nslab = len(parts)
    nc, lo, ex, ey, ez = field_extents(cfg, name)
    nzl = cfg.nz // nslab
    out = np.zeros((cfg.nz + 1, cfg.ny + 1, cfg.nx + 1, nc))
    sub = slab_config(cfg, nslab)
    for r, a in enumerate(parts):
        a = a.reshape(field_shape(sub, name)[:3] + (nc,))
        out[r * nzl:r * nzl + nzl + 1] = a[-lo:-lo + nzl + 1, -lo:-lo + cfg.ny + 1, -lo:-lo + cfg.nx + 1]
    return out


class _Dev:
    """A device array by address, for torch.as_tensor (CUDA array
    interface)."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3}


def _device_view(ptr: int, n: int, typestr: str, device):
    import torch
    return torch.as_tensor(_Dev(ptr, n, typestr), device=device)


class SlabGroup:
    """All slabs of a z decomposition in this process: contexts (on one GPU
    or several) stepped together, the exchange done by device copies."""

    def __init__(self, cfg: Config, eb: np.ndarray, p: np.ndarray | None, tp, nslab: int, outbox_cap: int,
                 capacity_factor: float = 1.25, devices=None, plasmas=None):
        """The particles of the whole grid as records (p, tp), or per slab a
        plasma description drawn on its device (plasmas[r], emsesg_load_plasma
        on the slab's grid; p None)."""
        self.cfg = cfg
        self.nslab = nslab
        self.sub = slab_config(cfg, nslab, capacity_factor)
        self.ctx = []
        for r in range(nslab):
            if devices is not None:
                import torch
                torch.cuda.set_device(devices[r])
            g = Emses(self.sub)
            if plasmas is not None:
                g.load_plasma(plasmas[r])
            else:
                pr, tpr = slab_particles(cfg, p, tp, r, nslab)
                g.upload_particles(pr, tpr)
            g.upload_field("eb", slab_field(cfg, eb, "eb", r, nslab))
            g.fx_load()
            g.fx_slab(True, outbox_cap)
            self.ctx.append(g)
        self.migrated = 0

    def close(self):
        for g in self.ctx:
            g.close()
        self.ctx = []

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def step(self, ustep: int = 2, do_sort: bool = False):
        import torch
        P, ns = self.nslab, self.cfg.nspec
        counts = [g.fx_slab_begin(ustep) for g in self.ctx]
        self.migrated += int(sum(c.sum() for c in counts))
        dev = torch.device("cuda")
        # arrivals: from below (the outbox of r - 1 upwards), then from above
        for r in range(P):
            up, dn = (r + 1) % P, (r - 1) % P
            for s in range(ns):
                for src, d in ((dn, 1), (up, 0)):
                    n = int(counts[src][s, d])
                    if n:
                        self.ctx[r].fx_slab_arrive(s + 1, self.ctx[src].fx_slab_outbox(s + 1, d), n)
        for g in self.ctx:
            g.fx_slab_border()
        # z border planes: sent up by r into r + 1's planes from below, sent
        # down by r into r - 1's planes from above
        for r in range(P):
            up, dn = (r + 1) % P, (r - 1) % P
            for src_which, dst, dst_which in ((1, up, 2), (0, dn, 3)):
                sr, nr, sj, nj = self.ctx[r].fx_slab_planes(src_which)
                dr, mr, dj, mj = self.ctx[dst].fx_slab_planes(dst_which)
                assert nr == mr and nj == mj
                _device_view(dr, mr, "<i8", dev).copy_(_device_view(sr, nr, "<i8", dev))
                _device_view(dj, mj, "<i8", dev).copy_(_device_view(sj, nj, "<i8", dev))
        torch.cuda.synchronize()
        for g in self.ctx:
            g.fx_slab_end(do_sort)

    def fields(self, name: str) -> np.ndarray:
        """rho or aj of the whole grid on its nodes 0..n."""
        return assemble(self.cfg, name, [g.download_field(name) for g in self.ctx])

    def counts(self) -> np.ndarray:
        return np.sum([g.fx_counts() for g in self.ctx], axis=0)


class ContextIO:
    """The slab-mode calls of a context with its buffers as torch tensors on
    its GPU (views of the device memory, no copies): what exchange_step
    needs from a slab."""

    def __init__(self, g: Emses, device=None):
        import torch
        self.g = g
        self.device = device if device is not None else torch.device("cuda", torch.cuda.current_device())

    def begin(self, ustep: int) -> np.ndarray:
        return self.g.fx_slab_begin(ustep)

    def outbox(self, spec: int, direction: int, n: int):
        return _device_view(self.g.fx_slab_outbox(spec, direction), n * REC_BYTES, "|u1", self.device)

    def planes(self, which: int):
        pr, nr, pj, nj = self.g.fx_slab_planes(which)
        return _device_view(pr, nr, "<i8", self.device), _device_view(pj, nj, "<i8", self.device)

    def new_records(self, n: int):
        import torch
        return torch.empty(n * REC_BYTES, dtype=torch.uint8, device=self.device)

    def arrive(self, spec: int, buf, n: int):
        self.g.fx_slab_arrive(spec, buf.data_ptr(), n)

    def border(self):
        self.g.fx_slab_border()

    def end(self, do_sort: bool):
        self.g.fx_slab_end(do_sort)

    def wait(self):
        import torch
        torch.cuda.synchronize(self.device)


class SlabRank:
    """One slab per process (rank r of P in a torch.distributed group, one
    GPU each): the exchange with the neighbours r - 1 and r + 1 (ring)
    through point-to-point sends and receives of device buffers."""

    def __init__(self, cfg: Config, eb: np.ndarray, p: np.ndarray, tp, outbox_cap: int, group=None,
                 capacity_factor: float = 1.25):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)
        if self.size < 2:
            raise ValueError("a slab decomposition needs two ranks or more")
        self.cfg = cfg
        self.sub = slab_config(cfg, self.size, capacity_factor)
        pr, tpr = slab_particles(cfg, p, tp, self.rank, self.size)
        self.g = Emses(self.sub)
        self.g.upload_particles(pr, tpr)
        self.g.upload_field("eb", slab_field(cfg, eb, "eb", self.rank, self.size))
        self.g.fx_load()
        self.g.fx_slab(True, outbox_cap)
        self.io = ContextIO(self.g)

    def close(self):
        self.g.close()

    def step(self, ustep: int = 2, do_sort: bool = False) -> np.ndarray:
        return exchange_step(self.io, self.dist, self.group, self.rank, self.size, ustep, do_sort)

    def totals(self) -> dict:
        """The run's global counters, summed over the ranks by one
        all-reduce: particles per species and escapes per species."""
        ns = self.sub.nspec
        local = np.concatenate([self.g.fx_counts()[:ns], self.g.get_counters().as_dict()["nesc"][:ns]])
        tot = reduce_counts(local, self.dist, self.group, self.io.device)
        return {"particles": tot[:ns], "nesc": tot[ns:]}


def reduce_counts(counts, dist, group=None, device=None) -> np.ndarray:
    """int64 counters summed over the ranks of `group` by one all-reduce
    (the global counts the reference reduces over its ranks: OhHelp's
    per-species totals, the escape counts)."""
    import torch
    a = np.asarray(counts, dtype=np.int64)
    t = torch.as_tensor(a.ravel().copy()).to(device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy().reshape(a.shape)


def exchange_step(io, dist, group, rank: int, size: int, ustep: int, do_sort: bool) -> np.ndarray:
    """One slab step of rank `rank` of `size` (size >= 2) with the exchange
    through torch.distributed point-to-point operations (all of a round's
    sends and receives posted together, so that no pairing can deadlock).
    `io` is the rank's slab (ContextIO, or any object with its methods).
    Returns the counts of the particles that left, [spec, dir]."""
    import torch
    up, dn = (rank + 1) % size, (rank - 1) % size
    counts = io.begin(ustep)
    ns = counts.shape[0]
    # 1. counts: mine to both neighbours, theirs back (neighbour below first)
    mine = torch.as_tensor(counts.ravel().copy(), dtype=torch.int64).to(io.device)
    from_dn = torch.empty_like(mine)
    from_up = torch.empty_like(mine)
    _p2p(dist, group, [(mine, up), (mine, dn)], [(from_dn, dn), (from_up, up)])
    c_dn = from_dn.cpu().numpy().reshape(ns, 2)
    c_up = from_up.cpu().numpy().reshape(ns, 2)
    # 2. records: each rank posts its sends and receives in the same order
    # (per species the outbox up, then down; receives from below, then from
    # above), so that with two ranks, where the neighbour below is the one
    # above, the messages still pair
    sends, recvs, below, above = [], [], [], []
    for s in range(ns):
        for d, peer in ((1, up), (0, dn)):
            n = int(counts[s, d])
            if n:
                sends.append((io.outbox(s + 1, d, n), peer))
        for src_counts, d, peer, dst in ((c_dn, 1, dn, below), (c_up, 0, up, above)):
            n = int(src_counts[s, d])
            if n:
                buf = io.new_records(n)
                recvs.append((buf, peer))
                dst.append((s, buf, n))
    _p2p(dist, group, sends, recvs)
    io.wait()
    # 3. arrivals of each species from below, then from above
    for s in range(ns):
        for lst in (below, above):
            for t, buf, n in lst:
                if t == s:
                    io.arrive(s + 1, buf, n)
    # 4. the x / y border exchange; 5. the z border planes (planes up, then
    # down; receives from below, then from above)
    io.border()
    sends, recvs = [], []
    for which, peer in ((1, up), (0, dn)):
        sends += [(t, peer) for t in io.planes(which)]
    for which, peer in ((2, dn), (3, up)):
        recvs += [(t, peer) for t in io.planes(which)]
    _p2p(dist, group, sends, recvs)
    io.wait()
    # 6. the rest of the step
    io.end(do_sort)
    return counts


def _p2p(dist, group, sends, recvs):
    ops = [dist.P2POp(dist.isend, t, _global(dist, group, peer), group) for t, peer in sends]
    ops += [dist.P2POp(dist.irecv, t, _global(dist, group, peer), group) for t, peer in recvs]
    if ops:
        for w in dist.batch_isend_irecv(ops):
            w.wait()


def _global(dist, group, rank: int) -> int:
    return rank if group is None else dist.get_global_rank(group, rank)
