"""Host logic of the ensemble runner: the seeded run draws, the graph block
length and the packing of runs into waves that fit device memory."""
import math

import numpy as np

from ctca_b200 import ensemble


def test_draws_follow_the_stated_ranges():
    cases = ensemble.ensemble_cases(512, seed=1005)
    assert len(cases) == 512
    sides = {c.n[0] for c in cases}
    assert sides == set(ensemble.SIDES)
    for c in cases:
        assert c.n[0] == c.n[1] == c.n[2]
        e, i = c.species
        assert 8 <= e.ppc <= 64 and 8 <= i.ppc <= 64
        assert 0.02 <= e.vth <= 0.1
        assert math.isclose(i.vth, e.vth / 10.0)
        assert math.isclose(i.qm / e.qm, -1.0 / 100.0)
        assert np.linalg.norm(c.b0) <= 0.3 + 1e-12
        assert c.e_modes == 4 and c.e_amp == 1e-3
    # seeded: the same draws again, other draws for another seed
    again = ensemble.ensemble_cases(512, seed=1005)
    assert [(c.n, c.species[0].ppc, c.b0) for c in cases] == [(c.n, c.species[0].ppc, c.b0) for c in again]
    other = ensemble.ensemble_cases(512, seed=1006)
    assert [c.b0 for c in cases] != [c.b0 for c in other]
    # about 3.1 G particles over the 512 runs
    total = sum(ensemble.particles(c) for c in cases)
    assert 2.0e9 < total < 4.5e9


def test_block_steps_is_a_common_multiple():
    assert ensemble.block_steps([1]) == 2
    assert ensemble.block_steps([1, 2, 4]) == 8
    assert ensemble.block_steps([2, 3]) == 12


def test_waves_fit_the_budget_and_cover_every_run():
    cases = ensemble.ensemble_cases(64, seed=9)
    budget = 8 << 30
    plan = ensemble.waves(cases, budget)
    seen = sorted(i for w in plan for i in w)
    assert seen == list(range(64))
    for w in plan:
        assert len(w) == 1 or sum(ensemble.run_bytes(cases[i]) for i in w) <= budget
