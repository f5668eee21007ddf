"""Exact FP64 operation count of one SSP-RK3 step per cell-update, from the
counting build of the oracle (oracle/gdf_oracle_count.cpp): the reference's
loops as the oracle restates them (structurally zero modal terms left out),
each + - * / and square root counted once.

MEASUREMENT INFRASTRUCTURE ONLY (runs the oracle, single-threaded).

    python oracle/count_flops.py [--out FILE]

Counts one step after `prepare` and one warm-up step on the Orszag-Tang
vortex at 128^2 (HLL, every cell limited), the rotor at 512^2 and the blast
at 512^2 (HLLD, sticky KXRCF + TVB, positivity limiter, face-B minmod)."""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "freljord-cfd-arsenal_b200"))

from gdf._abi import PROB_BLAST, PROB_ORSZAG_TANG, PROB_ROTOR, problem_config  # noqa: E402
from oracle import Oracle  # noqa: E402

CASES = (("orszag_tang", PROB_ORSZAG_TANG, 128), ("rotor", PROB_ROTOR, 512), ("blast", PROB_BLAST, 512))


def count(problem: int, n: int) -> dict:
    cfg, tend = problem_config(problem, n, n)
    o = Oracle(cfg, counting=True)
    uh, bx, by = o.init_data(problem)
    o.prepare(uh, bx, by)
    t, _, _ = o.step(uh, bx, by, 0.0, tend)
    o.reset_flops()
    t0 = time.perf_counter()
    o.step(uh, bx, by, t, tend)
    el = time.perf_counter() - t0
    add, mul, div, sq, pw = o.flops()
    cells = n * n
    tot = add + mul + div + sq
    return {"grid": [n, n], "flop_per_cell_update": tot / cells, "add_sub": add / cells, "mul": mul / cells,
            "div": div / cells, "sqrt": sq / cells, "other_calls": pw / cells, "seconds": el}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    res = {name: count(p, n) for name, p, n in CASES}
    text = json.dumps(res, indent=1)
    print(text)
    if a.out:
        with open(a.out, "w") as f:
            f.write(text + "\n")


if __name__ == "__main__":
    main()
