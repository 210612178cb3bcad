"""Shared builders for the parity tests (small cases the oracle runs in
seconds)."""
import numpy as np

from ctca_b200 import inputs
from ctca_b200.emses import PARTICLE_DTYPE


def case(n=(8, 8, 8), ppc=(6, 6), seed=11, b0=(0.0, 0.0, 0.2), e=True, vth_scale=1.0, npbnd=(0, 0, 0),
         nfbnd=(0, 0, 0), tile=(0, 0, 0)):
    c = inputs.workload_case(1)
    c.n = tuple(n)
    c.species[0].ppc, c.species[1].ppc = ppc
    c.species[0].vth *= vth_scale
    c.species[1].vth *= vth_scale
    for s in c.species:
        s.npbnd = tuple(npbnd)
    c.nfbnd = tuple(nfbnd)
    c.kmax = 2 * np.pi / min(n) * 2
    c.seed = seed
    c.b0 = b0
    c.sort_tile = tuple(tile)
    if not e:
        c.e_modes = 0
        c.e0 = (0.0, 0.0, 0.0)
    return c


def build(c, capacity_factor=1.0):
    c.capacity_factor = capacity_factor
    cfg = inputs.make_config(c)
    eb = inputs.make_fields(c)
    p, tp = inputs.make_particles(c)
    return cfg, eb, p, tp


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def same_particles(a, b):
    """Bit-exact equality of two particle buffers (all 64 bytes)."""
    return np.array_equal(np.ascontiguousarray(a).view(np.uint8), np.ascontiguousarray(b).view(np.uint8))


def particles_from(records):
    out = np.zeros(len(records), dtype=PARTICLE_DTYPE)
    for m, r in enumerate(records):
        for k, v in r.items():
            out[k][m] = v
    return out
