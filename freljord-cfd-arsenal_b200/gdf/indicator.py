"""Training data, training, thresholds and evaluation of the learned
troubled-cell indicator (no counterpart in the reference, which uses
KXRCF_Detector.f90 alone).

Data. Seeded MHD blasts (centre uniform in [-0.2, 0.2]^2, radius 0.1,
rho = 1, outer pressure 0.1, inner/outer pressure ratio log-uniform in
[1e2, 1e4], |B| uniform in [0, 100/sqrt(4 pi)] at a uniform angle, gamma
1.4, HLLD, KXRCF + TVB + positivity limiter) run on the device with the
plain solver. At sampled steps the state u before the step is kept, its
stage-1 pre-limit state u + dt L(u) is formed (Lh, LhEz and calculate_dt
through the C ABI, value for value the step's own), each interior cell
gets its 90 inputs (gdf_features of that state), and the step is then
taken by the plain solver, whose flag word gives the label

    y = the plain method changed the cell at stage 1
        (sticky KXRCF flag AND the characteristic TVB limiter modified it).

A gate that fires exactly on these cells reproduces the plain step: a
gated cell that TVB leaves alone and an ungated cell are the same.

Gate. With thresholds t_lo <= t_hi the limiter runs where p >= t_hi, not
where p < t_lo, and KXRCF (per stage) decides in between; (0, 0) is the
all-cells limiter and (0, > 1) is per-stage KXRCF exactly. The positivity
limiter and the divergence-free reconstruction always run unchanged in
FP64.

Run as a module:
    python -m gdf.indicator train --out weights.npz   (data, training, thresholds)
    python -m gdf.indicator eval --weights weights.npz --n 512 --seeds 1001 1002
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

import numpy as np

from . import (DETECT_ALL, DETECT_KXRCF, DETECT_LEARNED, NFEAT, PROB_BLAST, Mlp, Solver, init_data,
               problem_config)

WEIGHTS = os.path.join(os.path.dirname(__file__), "data", "indicator_blast256.npz")
STAGE_CHANGE = 0xFFFFFF       # per-stage change masks of the flag word
GATE_BIT = 1 << 24            # stage-1 gate bit of the flag word


def blast_params(seed: int) -> np.ndarray:
    """init_data parameters (cx, cy, r0, p_in, p_out, rho, Bx, By) of the
    seeded blast."""
    rng = np.random.default_rng(seed)
    cx, cy = rng.uniform(-0.2, 0.2, 2)
    ratio = math.exp(rng.uniform(math.log(1e2), math.log(1e4)))
    bmag = rng.uniform(0.0, 100.0 / math.sqrt(4 * math.pi))
    ang = rng.uniform(0.0, 2 * math.pi)
    p_out = 0.1
    return np.array([cx, cy, 0.1, p_out * ratio, p_out, 1.0, bmag * math.cos(ang), bmag * math.sin(ang)])


def blast_setup(n: int, seed: int, detector: int = DETECT_KXRCF, sticky: int = 1, exact: bool = True,
                params=None):
    """Config and initial state of the seeded blast on n x n cells (params
    "default": the benchmark blast, p = 1000 inside r = 0.1 at the centre,
    Bx = By = 100/sqrt(8 pi))."""
    cfg, tend = problem_config(PROB_BLAST, n, n)
    cfg.detector = detector
    cfg.kxrcf_sticky = sticky
    prm = None if params == "default" else (blast_params(seed) if params is None else params)
    uh, bx, by = init_data(cfg, PROB_BLAST, prm, exact=exact)
    return cfg, tend, uh, bx, by


class Labeller:
    """Stage-1 pre-limit states, their inputs and labels, on one grid size."""

    def __init__(self, cfg, exact: bool = True):
        a = cfg.copy()
        a.detector = DETECT_ALL
        k = cfg.copy()
        k.detector = DETECT_KXRCF
        k.kxrcf_sticky = 0
        self.s_all = Solver(a, exact)
        self.s_kx = Solver(k, exact)

    def prelimit(self, uh, bx, by):
        """u + dt L(u) for a state whose ghost cells are set (RK3.f90:60-100)."""
        s = self.s_all
        du = s.lh(uh)
        d1, d2 = s.lhez(uh)
        dt = s.dt(uh)
        return uh + dt * du, bx + dt * d1, by + dt * d2

    def sample(self, uh, bx, by):
        """(X [ncell, 90] float32, y [ncell] bool, kxrcf [ncell] bool,
        change [ncell] bool) of the stage-1 pre-limit state of uh."""
        ui, bi, ci = self.prelimit(uh, bx, by)
        X = self.s_all.features(ui)
        fa = self.s_all.limit(ui.copy(), bi.copy(), ci.copy()).ravel()
        fk = self.s_kx.limit(ui.copy(), bi.copy(), ci.copy()).ravel()
        change = (fa & STAGE_CHANGE) != 0
        kx = (fk & GATE_BIT) != 0
        return X, change & kx, kx, change


def collect(n: int, seeds, samples_per_run: int = 8, keep: float = 0.2, exact: bool = True, log=None):
    """Labelled cells from seeded blasts of n x n cells along the plain
    trajectory: a seeded `keep` share of each sample's cells."""
    Xs, ys = [], []
    lab = None
    for seed in seeds:
        cfg, tend, uh, bx, by = blast_setup(n, seed, exact=exact)
        if lab is None:
            lab = Labeller(cfg, exact)
        s = Solver(cfg, exact)
        s.upload(uh, bx, by)
        s.prepare()
        rng = np.random.default_rng(10_000 + seed)
        try:
            for k in range(samples_per_run):
                s.advance(tend * (k + 0.5) / samples_per_run, 10**7)
                X, y = plain_step_sample(s, lab, tend)
                sel = rng.random(y.size) < keep
                Xs.append(X[sel])
                ys.append(y[sel].astype(np.float32))
        except Exception as e:   # a run the plain method cannot finish keeps its samples so far
            if log:
                log(f"seed {seed}: stopped ({e})")
        s.close()
        if log:
            log(f"seed {seed}: {sum(len(v) for v in ys)} samples so far, positives {sum(v.sum() for v in ys):.0f}")
    return np.concatenate(Xs), np.concatenate(ys)


def plain_step_sample(s: Solver, lab: Labeller, tend: float):
    """Inputs of the stage-1 pre-limit state of s's current state and the
    plain method's stage-1 change flags, taking that step on s."""
    u, b, c = s.download()
    ui, _, _ = lab.prelimit(u, b, c)
    X = lab.s_all.features(ui)
    _, _, f = s.step(tend)
    return X, (f.ravel() & 0xFF) != 0


def choose_thresholds(p, y, miss: float = 0.01, fp: float | None = None):
    """t_lo: the largest threshold that leaves at most `miss` of the
    positives below it. t_hi: with fp None, t_lo (a single threshold, no
    KXRCF band); else the smallest threshold passing at most `fp` of the
    negatives above it (t_hi >= t_lo)."""
    y = y > 0.5
    pp = np.sort(p[y])
    pn = np.sort(p[~y])
    t_lo = float(pp[int(math.floor(miss * len(pp)))]) if len(pp) else 1.0
    if fp is None:
        return t_lo, t_lo
    t_hi = float(pn[min(len(pn) - 1, int(math.ceil((1 - fp) * len(pn))))]) if len(pn) else 0.0
    return t_lo, max(t_hi, t_lo)


MISS_TARGETS = (0.005, 0.01, 0.02, 0.05)


def train(X, y, seed: int = 0, epochs: int = 40, batch: int = 2048, lr: float = 2e-3, exact: bool = True,
          val_frac: float = 0.1, log=None):
    """Train on the device (the library's forward, backward and Adam
    kernels); returns (net, t_lo, t_hi, report). The shipped gate is a
    KXRCF band: t_lo the threshold that leaves 0.5% of the validation
    positives below it, t_hi the one that leaves 2%; the network decides
    outside the band and KXRCF, the reference's detector, inside it. The
    report lists the single thresholds for every miss target and the
    false-positive band setting."""
    rng = np.random.default_rng(seed)
    order = rng.permutation(len(y))
    nval = int(val_frac * len(y))
    iv, it = order[:nval], order[nval:]
    pos = float(y[it].sum())
    pos_weight = float((len(it) - pos) / max(pos, 1.0))
    net = Mlp(seed, exact)
    t0 = time.time()
    losses = net.train(X[it], y[it], epochs=epochs, batch=batch, lr=lr, pos_weight=pos_weight, seed=seed)
    t_train = time.time() - t0
    pv = net.predict(X[iv])
    yv = y[iv] > 0.5
    table = {}
    for m in MISS_TARGETS:
        t, _ = choose_thresholds(pv, yv, m)
        table[f"miss{m}"] = {"t_lo": t, "t_hi": t, "val_gated_share": float(np.mean(pv >= t)),
                             "val_fp_rate": float(np.mean(pv[~yv] >= t)) if (~yv).any() else 0.0}
    lo_b, hi_b = choose_thresholds(pv, yv, 0.01, 0.02)
    table["band"] = {"t_lo": lo_b, "t_hi": hi_b, "val_band_share": float(np.mean((pv >= lo_b) & (pv < hi_b)))}
    t_lo, t_hi = table["miss0.005"]["t_lo"], table["miss0.02"]["t_lo"]
    rep = {"samples": int(len(y)), "positives": int(y.sum()), "pos_weight": pos_weight,
           "epochs": epochs, "epoch_loss": [float(v) for v in losses], "train_s": t_train,
           "val_accuracy_at_0.5": float(np.mean((pv >= 0.5) == yv)), "t_lo": t_lo, "t_hi": t_hi,
           "thresholds": table}
    if log:
        log(json.dumps(rep))
    return net, t_lo, t_hi, rep


def save(path: str, net: Mlp, t_lo: float, t_hi: float, report: dict) -> None:
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    np.savez(path, params=net.params(), t_lo=np.float32(t_lo), t_hi=np.float32(t_hi),
             report=json.dumps(report))


def load_net(path: str = WEIGHTS, exact: bool = True):
    """(net, t_lo, t_hi) from a saved indicator."""
    z = np.load(path)
    net = Mlp(0, exact)
    net.set_params(z["params"])
    return net, float(z["t_lo"]), float(z["t_hi"])


def run(n: int, seed: int, net=None, t_lo=0.5, t_hi=0.5, exact: bool = True, tend=None, max_steps=10**7,
        params=None, detector=None, sticky: int = 1):
    """Seeded blast to tend with the plain method (net None: KXRCF, sticky,
    as the reference; or `detector`) or the learned gate; returns (uh,
    steps, ms per step, mean cells flagged in a step)."""
    det = (DETECT_KXRCF if detector is None else detector) if net is None else DETECT_LEARNED
    cfg, te, uh, bx, by = blast_setup(n, seed, det, sticky=sticky, exact=exact, params=params)
    s = Solver(cfg, exact)
    if net is not None:
        s.set_indicator(net, t_lo, t_hi)
    s.upload(uh, bx, by)
    s.prepare()
    t_end = te if tend is None else tend
    steps, ms = 0, 0.0
    gated, chunks = 0, 0
    while s.t < t_end and steps < max_steps:
        _, k, dms = s.advance_timed(t_end, min(200, max_steps - steps))
        if k == 0:
            break
        steps += k
        ms += dms
        gated += s.diagnostics()[3]
        chunks += 1
    u, _, _ = s.download()
    s.close()
    return u, steps, ms / max(steps, 1), gated / max(chunks, 1)


def fine_reference(n: int, seed: int, factor: int = 2, cache: str | None = None, exact: bool = True):
    """Cell-mean density of the plain run on a grid `factor` times finer,
    averaged onto n x n (cached as .npy under `cache`)."""
    path = os.path.join(cache, f"blast_ref_{n}x{factor}_seed{seed}.npy") if cache else None
    if path and os.path.exists(path):
        return np.load(path)
    u_f, _, _, _ = run(n * factor, seed, exact=exact)
    r = u_f[0, 0, 1:-1, 1:-1]
    k = factor
    rho = r.reshape(n, k, n, k).mean(axis=(1, 3))
    if path:
        os.makedirs(cache, exist_ok=True)
        np.save(path, rho)
    return rho


def evaluate(net, settings, n: int, seeds, ref_factor: int = 2, samples: int = 4, exact: bool = True,
             cache: str | None = None, log=None):
    """Held-out evaluation of gate settings {name: (t_lo, t_hi)}: per seed,
    the L1 density error of the plain run and of each learned run against a
    plain run on a grid ref_factor times finer, the L1 difference learned
    vs plain, whole-run device time of both, and each gate's miss /
    false-positive rates against the plain method's stage-1 decisions along
    the plain trajectory."""
    out = []
    for seed in seeds:
        u_p, st_p, ms_p, g_p = run(n, seed, None, exact=exact)
        rho_p = u_p[0, 0, 1:-1, 1:-1]
        rho_f = fine_reference(n, seed, ref_factor, cache, exact) if ref_factor else None
        rec = {"seed": seed, "n": n, "plain": {"steps": st_p, "ms_per_step": ms_p, "run_ms": ms_p * st_p,
                                               "flagged_per_step": g_p}}
        if rho_f is not None:
            rec["plain"]["l1_err"] = float(np.abs(rho_p - rho_f).mean())
        # gate quality along the plain trajectory
        cfg, tend, uh, bx, by = blast_setup(n, seed, exact=exact)
        lab = Labeller(cfg, exact)
        s = Solver(cfg, exact)
        s.upload(uh, bx, by)
        s.prepare()
        P, Y, KX = [], [], []
        for k in range(samples):
            s.advance(tend * (k + 0.5) / samples, 10**7)
            u, b, c = s.download()
            ui, bi, ci = lab.prelimit(u, b, c)
            X = lab.s_all.features(ui)
            KX.append((lab.s_kx.limit(ui.copy(), bi.copy(), ci.copy()).ravel() & GATE_BIT) != 0)
            _, _, f = s.step(tend)
            Y.append((f.ravel() & 0xFF) != 0)
            P.append(net.predict(X))
        s.close()
        P, Y, KX = np.concatenate(P), np.concatenate(Y), np.concatenate(KX)
        rec["positive_share"] = float(Y.mean())
        for name, (lo, hi) in settings.items():
            gate = (P >= hi) | ((P >= lo) & KX)
            try:
                u_l, st_l, ms_l, g_l = run(n, seed, net, lo, hi, exact=exact)
            except Exception as e:   # the learned run failed (e.g. lost positivity)
                rec[name] = {"t_lo": lo, "t_hi": hi, "failed": str(e),
                             "miss_rate": float(np.mean(~gate[Y])) if Y.any() else 0.0,
                             "false_positive_rate": float(np.mean(gate[~Y])) if (~Y).any() else 0.0}
                continue
            rho_l = u_l[0, 0, 1:-1, 1:-1]
            r = {"t_lo": lo, "t_hi": hi, "steps": st_l, "ms_per_step": ms_l, "run_ms": ms_l * st_l,
                 "speedup_run": ms_p * st_p / (ms_l * st_l), "flagged_per_step": g_l,
                 "l1_rho_vs_plain": float(np.abs(rho_l - rho_p).mean() / np.abs(rho_p).mean()),
                 "miss_rate": float(np.mean(~gate[Y])) if Y.any() else 0.0,
                 "false_positive_rate": float(np.mean(gate[~Y])) if (~Y).any() else 0.0,
                 "gated_share": float(gate.mean()), "band_share": float(np.mean((P >= lo) & (P < hi)))}
            if rho_f is not None:
                r["l1_err"] = float(np.abs(rho_l - rho_f).mean())
                r["l1_err_ratio"] = r["l1_err"] / rec["plain"]["l1_err"]
            rec[name] = r
        if log:
            log(json.dumps(rec))
        out.append(rec)
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m gdf.indicator")
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--n", type=int, nargs="+", default=[256],
                   help="grid sides; with several, --seeds gives the seed count of each")
    t.add_argument("--seeds", type=int, nargs="+", default=[32])
    t.add_argument("--samples-per-run", type=int, default=8)
    t.add_argument("--keep", type=float, default=0.2)
    t.add_argument("--epochs", type=int, default=40)
    t.add_argument("--out", default=WEIGHTS)
    e = sub.add_parser("eval")
    e.add_argument("--weights", default=WEIGHTS)
    e.add_argument("--n", type=int, default=512)
    e.add_argument("--seeds", type=int, nargs="+", default=[1001, 1002])
    e.add_argument("--ref-factor", type=int, default=2)
    e.add_argument("--all-settings", action="store_true", help="also every threshold of the training report")
    e.add_argument("--only", nargs="+", default=None, help="with --all-settings: these report entries only")
    e.add_argument("--out", default=None)
    e.add_argument("--cache", default=None, help="directory for the fine-grid reference densities")
    a = ap.parse_args(argv)
    log = lambda m: print(m, flush=True)  # noqa: E731
    if a.cmd == "train":
        t0 = time.time()
        if len(a.seeds) != len(a.n):
            raise SystemExit("--seeds needs one count per --n")
        parts = []
        for k, (n, ns) in enumerate(zip(a.n, a.seeds)):
            # disjoint training seeds per resolution (held-out seeds are 1000+)
            parts.append(collect(n, range(100 * k, 100 * k + ns), a.samples_per_run, a.keep, log=log))
        X = np.concatenate([p[0] for p in parts])
        y = np.concatenate([p[1] for p in parts])
        log(f"collected {len(y)} cells ({int(y.sum())} positive) in {time.time() - t0:.1f} s")
        net, t_lo, t_hi, rep = train(X, y, epochs=a.epochs, log=log)
        rep.update({"grid": a.n, "train_seeds": a.seeds, "samples_per_run": a.samples_per_run, "keep": a.keep})
        save(a.out, net, t_lo, t_hi, rep)
        log(f"saved {a.out}")
    else:
        net, t_lo, t_hi = load_net(a.weights)
        settings = {"shipped": (t_lo, t_hi)}
        if a.all_settings:
            rep = json.loads(str(np.load(a.weights)["report"]))
            for k, v in rep.get("thresholds", {}).items():
                if a.only is None or k in a.only:
                    settings[k] = (v["t_lo"], v["t_hi"])
        res = evaluate(net, settings, a.n, a.seeds, a.ref_factor, cache=a.cache, log=log)
        if a.out:
            with open(a.out, "w") as f:
                json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
