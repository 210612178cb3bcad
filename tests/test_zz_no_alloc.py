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


def run_noalloc(lib, stream, p, n):
    import torch

    buf = p.view(np.uint8).copy() if p.size else np.zeros(64, dtype=np.uint8)
    d_in = torch.from_numpy(buf).cuda()
    d_out = torch.full_like(d_in, 0xAB)
    d_kept = torch.full((1,), -7, dtype=torch.int64, device="cuda")
    rc = lib.emsesg_compact_noalloc(ctypes.c_void_p(d_in.data_ptr()), n, ctypes.c_void_p(d_out.data_ptr()),
                                    ctypes.c_void_p(d_kept.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
    assert rc == 0
    torch.cuda.synchronize()
    kept = int(d_kept.item())
    return d_out[: kept * 64].cpu().numpy().view(PARTICLE_DTYPE), kept


def test_compact_noalloc_matches_compact_in_a_row(gpu):
    """Calls in a row through the shared scratch: 256,000 particles (a partial
    last tile), exactly the maximum 2^20, none, all dropped, and 4097 (one
    particle into a second tile) -- each equal to emsesg_compact."""
    import torch

    lib = load_library()
    stream = torch.cuda.current_stream()
    # (cells, ppc, seed, drop one in `every` (0: drop all), keep the first `take`)
    trials = [((40, 40, 40), 4, 21, 3, None), ((64, 64, 64), 4, 22, 5, None), ((8, 8, 8), 2, 23, 2, 0),
              ((16, 16, 16), 2, 24, 0, None), ((20, 20, 20), 1, 25, 7, 4097)]
    for n_cells, ppc, seed, every, take in trials:
        cfg, p, tp = one_species(n_cells, ppc, seed)
        if take is not None:
            p, tp = p[:take].copy(), np.array([take], dtype=np.int64)
        assert p.size <= MAX_PARTICLES
        rng = np.random.default_rng(seed)
        if every:
            p["nid"][rng.random(p.size) < 1.0 / every] = -1
        else:
            p["nid"] = -1
        got, kept = run_noalloc(lib, stream, p, p.size)
        assert kept == int((p["nid"] != -1).sum())
        if p.size == 0:
            assert kept == 0
            continue
        ref, ref_kept = existing_compact(cfg, p, tp)
        assert kept == ref_kept
        assert np.array_equal(got.view(np.uint8), ref.view(np.uint8))


def test_compact_noalloc_rejects_bad_arguments(gpu):
    lib = load_library()
    dummy = ctypes.c_void_p(16)  # never dereferenced: the argument checks come first
    assert lib.emsesg_compact_noalloc(dummy, MAX_PARTICLES + 1, ctypes.c_void_p(1 << 30), ctypes.c_void_p(8),
                                      None) == ERR_ARG
    assert lib.emsesg_compact_noalloc(dummy, 8, dummy, ctypes.c_void_p(8), None) == ERR_ARG  # d_out == d_in
    base = 1 << 30
    n = 100  # 6400 bytes
    # output overlapping the input's tail, and the count inside the input or the output
    assert lib.emsesg_compact_noalloc(ctypes.c_void_p(base), n, ctypes.c_void_p(base + 64 * 50),
                                      ctypes.c_void_p(base + (1 << 20)), None) == ERR_ARG
    assert lib.emsesg_compact_noalloc(ctypes.c_void_p(base), n, ctypes.c_void_p(base + (1 << 20)),
                                      ctypes.c_void_p(base + 64 * 10), None) == ERR_ARG
    assert lib.emsesg_compact_noalloc(ctypes.c_void_p(base), n, ctypes.c_void_p(base + (1 << 20)),
                                      ctypes.c_void_p(base + (1 << 20) + 8), None) == ERR_ARG
