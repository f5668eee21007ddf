"""The counting build of the oracle (oracle/gdf_oracle_count.cpp, the same
source on the counting scalar of flopcount.h) computes the same values as
the oracle, so its tally is the operation count of the oracle's own step;
the tally is deterministic and covers every operation kind."""
import numpy as np
import pytest

import gdf
from oracle import Oracle


@pytest.mark.parametrize("problem", [gdf.PROB_ORSZAG_TANG, gdf.PROB_ROTOR, gdf.PROB_BLAST])
def test_counting_oracle_matches_oracle_and_counts(problem):
    cfg, tend = gdf.problem_config(problem, 20, 16)
    states, counts = [], []
    for counting in (False, True, True):
        o = Oracle(cfg, counting=counting)
        uh, bx, by = o.init_data(problem)
        o.prepare(uh, bx, by)
        t, _, _ = o.step(uh, bx, by, 0.0, tend)
        if counting:
            o.reset_flops()
        t, dt, f = o.step(uh, bx, by, t, tend)
        states.append((uh, bx, by, f, dt))
        if counting:
            counts.append(o.flops())
    for a, b in zip(states[0], states[1]):
        assert np.array_equal(a, b)
    assert counts[0] == counts[1]
    add, mul, div, sq, _ = counts[0]
    cells = cfg.nx * cfg.ny
    assert add > 1e4 * cells and mul > 1e4 * cells and div > 1e3 * cells and sq > 10 * cells
