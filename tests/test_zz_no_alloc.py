"""emsesg_compact_noalloc, the compaction for hosts that cannot allocate
device memory (their device arrays come from their own pool or framework),
against the existing emsesg_compact entry point, through the C ABI.

The new entry point takes device buffers the caller owns and uses only its
fixed file-scope scratch; two calls in a row with different data must both
match emsesg_compact bit for bit (the scratch keeps the previous call's
contents and must not leak into the next result).  This file is collected
last so that a failure here does not stop the other tests."""
import ctypes

import numpy as np
import pytest

from ctca_b200 import inputs
from ctca_b200.emses import ERR_ARG, PARTICLE_DTYPE, Emses, load_library

from helpers import case

pytestmark = pytest.mark.gpu

MAX_PARTICLES = 1 << 20  # EMSESG_NOALLOC_MAX_PARTICLES


def one_species(n_cells, ppc, seed):
    c = case(n=n_cells, ppc=(ppc, ppc), seed=seed)
    c.species = [c.species[0]]
    cfg = inputs.make_config(c)
    p, tp = inputs.make_particles(c)
    return cfg, p, tp


def existing_compact(cfg, p, tp):
    g = Emses(cfg)
    g.upload_particles(p, tp)
    kept = g.compact(1)
    out, _ = g.download_particles()
    g.close()
    return out, int(kept[0])


def test_compact_noalloc_matches_compact_twice(gpu):
    import torch

    lib = load_library()
    stream = torch.cuda.current_stream()
    trials = [((40, 40, 40), 4, 21, 3), ((64, 64, 64), 4, 22, 5)]  # 256,000 and 1,048,576 particles
    for n_cells, ppc, seed, every in trials:
        cfg, p, tp = one_species(n_cells, ppc, seed)
        assert p.size <= MAX_PARTICLES
        rng = np.random.default_rng(seed)
        p["nid"][rng.random(p.size) < 1.0 / every] = -1
        d_in = torch.from_numpy(p.view(np.uint8).copy()).cuda()
        d_out = torch.full_like(d_in, 0xAB)
        d_kept = torch.full((1,), -7, dtype=torch.int64, device="cuda")
        rc = lib.emsesg_compact_noalloc(ctypes.c_void_p(d_in.data_ptr()), p.size, ctypes.c_void_p(d_out.data_ptr()),
                                        ctypes.c_void_p(d_kept.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0
        torch.cuda.synchronize()
        kept = int(d_kept.item())
        got = d_out[: kept * 64].cpu().numpy().view(PARTICLE_DTYPE)
        ref, ref_kept = existing_compact(cfg, p, tp)
        assert kept == ref_kept == int((p["nid"] != -1).sum())
        assert np.array_equal(got.view(np.uint8), ref.view(np.uint8))


def test_compact_noalloc_rejects_oversize(gpu):
    lib = load_library()
    dummy = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    assert lib.emsesg_compact_noalloc(dummy, MAX_PARTICLES + 1, ctypes.c_void_p(32), dummy, None) == ERR_ARG
    assert lib.emsesg_compact_noalloc(dummy, 8, dummy, dummy, None) == ERR_ARG  # d_out == d_in
