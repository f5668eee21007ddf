"""The reference's main program (main.f90) on the B200 library:

    get_GLP + init_data   ->  problem_config + init_data
    RK3                   ->  Solver.prepare + the step loop, with the
                              Q*flash.txt / T.txt frames of RK3.f90 when
                              flash is on (frameMAX frames up to tend)
    save_XY               ->  save_xy
    save_solution         ->  save_solution
    calculate_L2error     ->  l2_error (meaningful for the vortex)

and the per-step print of RK3.f90 (t, umax, totaldiv) when verbose. Beyond
main.f90: stop after a number of steps, write a binary checkpoint at the
end, restart from one (value-exact continuation), skip the output files.

    python -m gdf.run --problem ot --n 128 --out out_dir [--flash] [--tend T]
    python -m gdf.run --problem rotor --n 512 --steps 200 --checkpoint r.ckpt --no-save
    python -m gdf.run --problem rotor --n 512 --restart r.ckpt --steps 1 --no-save
"""
from __future__ import annotations

import argparse
import os
import time

import numpy as np

from . import (PROB_BLAST, PROB_CLOUD_SHOCK, PROB_ORSZAG_TANG, PROB_ROTOR, PROB_VORTEX, Solver, init_data,
               l2_error, problem_config, save_frame, save_solution, save_xy)

PROBLEMS = {"vortex": PROB_VORTEX, "ot": PROB_ORSZAG_TANG, "rotor": PROB_ROTOR, "blast": PROB_BLAST,
            "cloud": PROB_CLOUD_SHOCK}


def run(problem: int, nx: int, ny: int, out: str, tend: float | None = None, flash: bool = False,
        frame_max: int = 200, exact: bool = True, verbose: bool = False, cfg=None, params=None,
        max_steps: int | None = None, checkpoint: str | None = None, restart: str | None = None,
        save: bool = True):
    """Run one problem to tend as main.f90 does; returns (t, steps, L2).
    max_steps stops earlier; checkpoint writes the final state (gdf_checkpoint_save);
    restart continues from a checkpoint of the same configuration instead of
    the initial data; save=False skips the output files (L2 is then None)."""
    if cfg is None:
        cfg, te = problem_config(problem, nx, ny)
    else:
        te = tend
    tend = te if tend is None else tend
    if save or flash:
        os.makedirs(out, exist_ok=True)
    s = Solver(cfg, exact)
    if restart:
        s.restore(restart)
    else:
        uh, bx, by = init_data(cfg, problem, params, exact=exact)
        s.upload(uh, bx, by)
        s.prepare()
    if verbose:
        umax, tdiv, _, _ = s.diagnostics()
        print(0.0, " ", umax, " ", tdiv)
    if flash:
        save_frame(cfg, s.download()[0], s.t, out, reset=True, exact=exact)
    tt = tend / frame_max
    countf = 1
    steps = 0
    while s.t < tend and (max_steps is None or steps < max_steps):
        t, dt, _ = s.step(tend, flags=False)
        steps += 1
        if verbose:
            umax, tdiv, _, _ = s.diagnostics()
            print(t, " ", umax, " ", tdiv)
        if flash and (t > tt * countf or t == tend):
            save_frame(cfg, s.download()[0], t, out, exact=exact)
            countf += 1
    if checkpoint:
        s.checkpoint(checkpoint)
    L2 = None
    if save:
        uh, _, _ = s.download()
        save_xy(cfg, out, exact=exact)
        t20 = tend if tend <= 5 else 0.0
        save_solution(cfg, uh, out, exact=exact)
        L2 = l2_error(cfg, uh, t20, exact=exact)
    s.close()
    return s.t, steps, L2


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m gdf.run")
    ap.add_argument("--problem", choices=sorted(PROBLEMS), default="ot")
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--ny", type=int, default=None)
    ap.add_argument("--tend", type=float, default=None)
    ap.add_argument("--out", default="gdf_out")
    ap.add_argument("--flash", action="store_true", help="write the Q*flash.txt frames")
    ap.add_argument("--frames", type=int, default=200)
    ap.add_argument("--fma", action="store_true", help="the FMA build")
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--steps", type=int, default=None, help="stop after this many steps")
    ap.add_argument("--checkpoint", default=None, help="write a checkpoint of the final state here")
    ap.add_argument("--restart", default=None, help="continue from this checkpoint")
    ap.add_argument("--no-save", action="store_true", help="write no output files")
    a = ap.parse_args(argv)
    t0 = time.time()
    t, steps, L2 = run(PROBLEMS[a.problem], a.n, a.ny or a.n, a.out, a.tend, a.flash, a.frames, not a.fma,
                       a.verbose, max_steps=a.steps, checkpoint=a.checkpoint, restart=a.restart,
                       save=not a.no_save)
    print(f"t = {t}  steps = {steps}  wall {time.time() - t0:.2f} s")
    if L2 is not None:
        print("L2", " ".join(f"{v:.6e}" for v in L2))


if __name__ == "__main__":
    main()
