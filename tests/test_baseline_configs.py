"""Parity of the product build with the CPU oracle on the benchmark
configurations themselves, through the C ABI:

  * Orszag-Tang 128^2 (init3.txt: HLL, TVB M = 50, CFL 0.15, periodic):
    the first 10 steps compared after every step, then both sides run on
    their own to t = 0.5 and the end states and flag words are compared
    (relative L1 per variable, printed, and flag sets);
  * rotor 512^2 (HLLD, sticky KXRCF + TVB, positivity limiter, face-B
    minmod): 3 steps, compared after every step;
  * blast 2048^2 (HLLD, sticky KXRCF + TVB, positivity limiter, face-B
    minmod, piecewise-constant start): 1 step.

The product build has no FMA contraction, so every value must be equal
(==, the tolerance of these tests), dt included, and the troubled-cell
words identical; the relative L1 of 1e-12 per variable per step the
benchmark asks for is reported beside."""
import numpy as np
import pytest

import gdf
from oracle import Oracle

pytestmark = pytest.mark.gpu


def rel_l1_per_var(a, b):
    d = np.abs(a - b)[:, :, 1:-1, 1:-1].sum(axis=(1, 2, 3))
    s = np.abs(b)[:, :, 1:-1, 1:-1].sum(axis=(1, 2, 3))
    return d / np.where(s > 0, s, s[0])


def start(problem, n):
    cfg, tend = gdf.problem_config(problem, n, n)
    o = Oracle(cfg)
    uh, bx, by = o.init_data(problem)
    s = gdf.Solver(cfg)
    s.upload(uh, bx, by)
    f_gpu = s.prepare()
    f_orc = o.prepare(uh, bx, by)
    assert np.array_equal(f_gpu, f_orc), "prepare: troubled-cell words differ"
    return cfg, tend, o, s, (uh, bx, by)


def compare(s, state, f_gpu, f_orc, what):
    ug, bxg, byg = s.download()
    uh, bx, by = state
    r = rel_l1_per_var(ug, uh)
    assert np.isfinite(ug).all(), f"{what}: non-finite state"
    assert np.array_equal(ug, uh), f"{what}: uh differs, relative L1 per variable {r}"
    assert np.array_equal(bxg, bx) and np.array_equal(byg, by), f"{what}: face B differs"
    assert np.array_equal(f_gpu, f_orc), f"{what}: troubled-cell words differ"
    return r


def test_orszag_tang_128_to_t05():
    cfg, tend, o, s, state = start(gdf.PROB_ORSZAG_TANG, 128)
    uh, bx, by = state
    t = 0.0
    for k in range(10):
        tg, dtg, fg = s.step(tend)
        t, dto, fo = o.step(uh, bx, by, t, tend)
        assert dtg == dto and tg == t, f"step {k + 1}: dt {dtg} vs {dto}"
        compare(s, state, fg, fo, f"OT 128^2 step {k + 1}")
    steps = 10
    while t < tend:
        t, _, fo = o.step(uh, bx, by, t, tend)
        steps += 1
    tg, ng = s.advance(tend, 10**6)
    assert tg == t and ng == steps - 10, f"GPU reached t={tg} in {ng + 10} steps, oracle t={t} in {steps}"
    ug, bxg, byg = s.download()
    r = rel_l1_per_var(ug, uh)
    print(f"\nOT 128^2 to t={t:.6f} in {steps} steps: relative L1 per variable {r.tolist()}, "
          f"flagged cells {int((fo != 0).sum())}")
    assert (r <= 1e-12).all()
    assert np.array_equal(ug, uh) and np.array_equal(bxg, bx) and np.array_equal(byg, by)


def test_rotor_512_three_steps():
    cfg, tend, o, s, state = start(gdf.PROB_ROTOR, 512)
    uh, bx, by = state
    t = 0.0
    for k in range(3):
        tg, dtg, fg = s.step(tend)
        t, dto, fo = o.step(uh, bx, by, t, tend)
        assert dtg == dto, f"step {k + 1}: dt {dtg} vs {dto}"
        r = compare(s, state, fg, fo, f"rotor 512^2 step {k + 1}")
        assert (r <= 1e-12).all()


def test_blast_2048_one_step():
    cfg, tend, o, s, state = start(gdf.PROB_BLAST, 2048)
    uh, bx, by = state
    tg, dtg, fg = s.step(tend)
    t, dto, fo = o.step(uh, bx, by, 0.0, tend)
    assert dtg == dto
    r = compare(s, state, fg, fo, "blast 2048^2 step 1")
    assert (r <= 1e-12).all()
