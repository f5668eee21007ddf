#!/usr/bin/env python
"""Benchmark of the B200 GDF P2 MHD step: P2 MHD cell-updates/s.

Workload: the MHD rotor at 512x512, P2 modal DG in FP64, HLLD flux, KXRCF
detector + characteristic TVB limiter with the face-B minmod + positivity
limiter, SSP-RK3 (the
plain method at scale). One step = one full SSP-RK3 step of the whole
grid (3 stages + limiters + div-free reconstruction + dt); one
cell-update = one cell advanced by one step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs one process per GPU under torchrun; each rank advances its own
replica of the workload (the path runs on one GPU; replicas only), timed
on the device and reported as the max over ranks. Prints one JSON line on
rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "freljord-cfd-arsenal_b200"))

METRIC = "P2 MHD cell-updates/s on 1 B200, learned-indicator vs plain at equal L1 err"
UNIT = "cell-updates/s"
NX = NY = 512
WORKLOAD = ("MHD rotor 512x512 on [0,1]^2, P2 modal DG FP64 (8 vars x 10 modal slots), HLLD flux, "
            "KXRCF detector + characteristic TVB (M=10) + face-B minmod + positivity limiter, corner-Ez "
            "CT + Balsara div-free B, SSP-RK3, CFL 0.15 (plain method)")

# Compulsory HBM bytes per cell for one launch of each kernel kind (FP64,
# 52 live modal slots = 416 B per cell state): what one launch must read
# and write at least, stage mean for the residual kernel.
ALG_BYTES_PER_CELL = {
    "face_x": 416 + 40 * 8 + 5 * 8,          # cell modes once, Fxhat + EzRL of the cell's face
    "face_y": 416 + 40 * 8 + 5 * 8,
    "vertex": 416 + 8,                       # cell modes once, one vertex Ez
    "cell": (1888 + 2 * 2304) / 3,           # U + faces' Fhat + U0/UI read, UI (+U0) written; stage mean
    "bface": 2 * (5 * 8 + 8 + 3 * 8 * 3),    # two faces: Ez points, vertex, B/B0/BI read+written
    "limit": 416 + 416 + 4,                  # pre-limit modes, limited modes, flag (face-B minmod on:
                                             # the div-free reconstruction is its own kernel)
    "limit_tvb": 416 + 416 + 4,              # per deferred (gated) cell: modes, limited modes, flag
    "faceb_limit": 8 * 8 + 2 * 4 * 8,        # 4 Bx + 4 By modes of the cell, 2 coefficients of its 2 faces r+w
    "divfree": 2 * 3 * 8 + 16 * 8,           # 3 coefficients of 2 owned faces, 16 B modes written
    "set_bc": 0.0,
    "dt": 8 * 8,                             # cell averages
}
# the limiter with the div-free reconstruction fused (face-B minmod off)
ALG_BYTES_LIMIT_FUSED = 416 + 2 * 6 * 8 + 416 + 4   # + 4 face polys (2 owned)


def read_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    except Exception:
        return 6650.0, "fallback"


def nvml_index(local: int):
    """NVML handle of this process's CUDA device: NVML numbers GPUs
    regardless of CUDA_VISIBLE_DEVICES, so follow its entry (an index or a
    GPU UUID) when it is set."""
    import pynvml
    vis = [v.strip() for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip()]
    if local < len(vis):
        v = vis[local]
        if v.startswith("GPU-"):
            return pynvml.nvmlDeviceGetHandleByUUID(v)
        if v.isdigit():
            return pynvml.nvmlDeviceGetHandleByIndex(int(v))
    return pynvml.nvmlDeviceGetHandleByIndex(local)


class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled through NVML every
    10 ms on a thread, each sample stamped; `mark()` brackets the timed
    region and only samples inside it count. Reading only: nothing is set.
    Falls back to `nvidia-smi -lms 100` when NVML is not importable."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4), ("hw_power_brake_slowdown", 0x80))

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.t = None
        self.stop_evt = threading.Event()
        self.samples: list[tuple] = []     # (time, sm MHz, max MHz, reasons bitmask)
        self.window = None
        self.source = None

    def start(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            h = nvml_index(self.device)
            smax = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)

            def poll():
                while not self.stop_evt.is_set():
                    try:
                        sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                        r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                        self.samples.append((time.perf_counter(), float(sm), float(smax), int(r)))
                    except Exception:
                        pass
                    time.sleep(0.01)
            self.source = "nvml"
            self.t = threading.Thread(target=poll, daemon=True)
            self.t.start()
            return
        except Exception:
            pass
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.source = "nvidia-smi"
            self.t = threading.Thread(target=self._read_smi, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read_smi(self):
        bits = dict(self.REASONS)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.proc.stdout:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                r = sum(bits[nm] for nm, v in zip(names, f[5:9]) if v.lower() == "active")
                self.samples.append((time.perf_counter(), float(f[1]), float(f[2]), r))
            except ValueError:
                continue

    def mark(self, t0: float, t1: float):
        """The host times that bracket the timed region."""
        self.window = (t0, t1)

    def stop(self) -> dict | None:
        self.stop_evt.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.t:
            self.t.join(timeout=2)
        if not self.samples:
            return None
        inside = self.samples
        if self.window:
            t0, t1 = self.window
            inside = [x for x in self.samples if t0 <= x[0] <= t1] or \
                [min(self.samples, key=lambda x: abs(x[0] - 0.5 * (t0 + t1)))]
        reasons = sorted({nm for _, _, _, r in inside for nm, b in self.REASONS if r & b})
        return {"sm_mhz": statistics.median(x[1] for x in inside), "sm_max_mhz": max(x[2] for x in inside),
                "reasons": reasons, "samples": len(inside), "source": self.source}


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def reduce_max_ms(ms: float, dist, device) -> float:
    """Max over ranks of the device-timed region (ms); identity on one rank."""
    if dist is None:
        return ms
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(world: int, steps: int, ms_max: float) -> float:
    """Whole-job cell-updates/s: every rank advances its own replica."""
    return world * NX * NY * steps / (ms_max / 1e3)


def make_state(gdf):
    cfg, _ = gdf.problem_config(gdf.PROB_ROTOR, NX, NY)
    uh, bx, by = gdf.init_data(cfg, gdf.PROB_ROTOR)
    return cfg, uh, bx, by


def cpu_baseline(gdf, steps: int):
    """The oracle (CPU restatement of the reference) on the same workload."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    from oracle import Oracle, set_threads
    cores = set_threads(0)
    cfg, uh, bx, by = make_state(gdf)
    o = Oracle(cfg)
    o.prepare(uh, bx, by)
    t, _, _ = o.step(uh, bx, by, 0.0, 1e9)          # warm-up step
    t0 = time.perf_counter()
    for _ in range(steps):
        t, _, _ = o.step(uh, bx, by, t, 1e9)
    el = time.perf_counter() - t0
    return {"value": NX * NY * steps / el, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"rotor {NX}x{NY} (the benchmark workload), {steps} timed steps after prepare and 1 "
                      f"warm-up step, oracle/gdf_oracle.cpp with OpenMP on {cores} host threads",
            "seconds": el}


def learned_blast(gdf, steps: int):
    """Plain (KXRCF) vs learned-indicator throughput on the MHD blast.

    Whole runs at 512^2 (t = 0.01, every step timed) give the throughput of
    both methods over the blast's evolution and the L1 density difference
    learned vs plain; at 2048^2, `steps` steps from the start of the run
    (after 3 warm-up steps) are timed for both."""
    from gdf.indicator import WEIGHTS, load_net, run
    import numpy as np
    net, lo, hi = load_net(WEIGHTS)
    out = {"weights": os.path.relpath(WEIGHTS, REPO), "t_lo": lo, "t_hi": hi}
    u_p, st_p, ms_p, g_p = run(512, 0, None, params="default")
    u_l, st_l, ms_l, g_l = run(512, 0, net, lo, hi, params="default")
    rho_p, rho_l = u_p[0, 0, 1:-1, 1:-1], u_l[0, 0, 1:-1, 1:-1]
    out["blast512_full_run"] = {
        "plain": {"value": 512 * 512 / (ms_p / 1e3), "ms_per_step": ms_p, "steps": st_p,
                  "gated_cells_per_step": g_p},
        "learned": {"value": 512 * 512 / (ms_l / 1e3), "ms_per_step": ms_l, "steps": st_l,
                    "gated_cells_per_step": g_l},
        "speedup": ms_p * st_p / (ms_l * st_l),
        "l1_rho_learned_vs_plain": float(np.abs(rho_l - rho_p).mean() / np.abs(rho_p).mean())}
    n = 2048
    res = {}
    for name, det in (("plain", gdf.DETECT_KXRCF), ("learned", gdf.DETECT_LEARNED)):
        cfg, tend = gdf.problem_config(gdf.PROB_BLAST, n, n)
        cfg.detector = det
        uh, bx, by = gdf.init_data(cfg, gdf.PROB_BLAST)
        s = gdf.Solver(cfg)
        if det == gdf.DETECT_LEARNED:
            s.set_indicator(net, lo, hi)
        s.upload(uh, bx, by)
        s.prepare()
        s.advance_timed(tend, 3)
        _, k, ms = s.advance_timed(tend, steps)
        res[name] = {"value": n * n * k / (ms / 1e3), "ms_per_step": ms / k, "steps": k}
        s.close()
    res["speedup"] = res["plain"]["ms_per_step"] / res["learned"]["ms_per_step"]
    out["blast2048_first_steps"] = res
    return out


def ensemble_bench(gdf, steps: int):
    """The 64-instance ensemble (Orszag-Tang / rotor / blast, sides 64..512,
    HLLD): the plain GPU path (one handle per instance, KXRCF, graph
    replays, instances one after another), the batched plain method, and
    the batched learned-indicator method (autotuned tile shape)."""
    from gdf.indicator import WEIGHTS, load_net
    net, lo, hi = load_net(WEIGHTS)
    items = gdf.ensemble_configs(64, 0)
    cells = [c.nx * c.ny for c, _, _, _ in items]
    states = [gdf.init_data(c, p, prm) for c, p, prm, _ in items]
    out = {"instances": len(items), "cells": int(sum(cells)), "sides": sorted({c.nx for c, _, _, _ in items})}
    # plain, one instance at a time
    cu, tot_ms = 0, 0.0
    for (c, p, prm, tend), st in zip(items, states):
        cp = c.copy()
        cp.detector = gdf.DETECT_KXRCF
        s = gdf.Solver(cp)
        s.upload(*st)
        s.prepare()
        s.advance_timed(tend, 3)
        _, k, ms = s.advance_timed(tend, steps)
        cu += k * cp.nx * cp.ny
        tot_ms += ms
        s.close()
    out["plain_sequential"] = {"value": cu / (tot_ms / 1e3), "ms_per_step": tot_ms / steps}
    for name, learned in (("batched_plain", False), ("batched_learned", True)):
        cfgs = []
        for c, _, _, _ in items:
            cc = c.copy()
            cc.detector = gdf.DETECT_LEARNED if learned else gdf.DETECT_KXRCF
            cfgs.append(cc)
        e = gdf.Ensemble(cfgs)
        if learned:
            e.set_indicator(net, lo, hi)
        for i, st in enumerate(states):
            e.upload(i, *st)
        e.prepare()
        for i, (_, _, _, tend) in enumerate(items):
            e.set_time(i, 0.0, tend)
        e.advance(2)
        tune_ms = e.tune(1)
        e.advance(1)
        l0 = e.kernel_launches()
        cu, act, ms = e.advance(steps)
        out[name] = {"value": cu / (ms / 1e3), "ms_per_step": ms / steps, "tiles": e.tiles(),
                     "launches_per_step": (e.kernel_launches() - l0) / steps,
                     "tuner_best_ms": float(min(x for x in tune_ms if x > 0))}
        e.close()
    out["speedup_batched_learned_vs_plain"] = out["batched_learned"]["value"] / out["plain_sequential"]["value"]
    return out


def run_reference(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    import gdf
    k = max(1, min(args.steps, 10))
    w = max(0, min(args.warmup, 1))
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    from oracle import Oracle, set_threads
    cores = set_threads(0)
    cfg, uh, bx, by = make_state(gdf)
    o = Oracle(cfg)
    o.prepare(uh, bx, by)
    t = 0.0
    for _ in range(w):
        t, _, _ = o.step(uh, bx, by, t, 1e9)
    t0 = time.perf_counter()
    for _ in range(k):
        t, _, _ = o.step(uh, bx, by, t, 1e9)
    el = time.perf_counter() - t0
    value = NX * NY * k / el
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": el / k * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "grid": [NX, NY], "problem": "rotor"},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{k} steps (of --steps {args.steps}) of the rotor {NX}x{NY} after prepare "
                                   f"and {w} warm-up step(s); the reference Fortran cannot be built here "
                                   "(no Fortran compiler), so its CPU restatement oracle/gdf_oracle.cpp runs"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_quick(args):
    """Warm-up and timed steps only: the commands the ncu captures run.

    --workload rotor           the benchmark workload (rotor 512^2, plain)
    --workload blast-learned   blast 512^2 with the shipped learned gate
    --workload ensemble-small  8 instances (64^2..160^2, OT / rotor / blast,
                               HLLD, learned gate) in the persistent kernels
    --workload mlp-train       one epoch of indicator training on 65536
                               synthetic samples (batch 2048)"""
    import gdf
    gdf.set_device(dist_env()[2])
    w = args.workload
    if w == "rotor":
        cfg, uh, bx, by = make_state(gdf)
        s = gdf.Solver(cfg, exact=not args.fma)
        s.upload(uh, bx, by)
        s.prepare()
        if args.warmup:
            s.advance_timed(1e9, args.warmup)
        _, n, ms = s.advance_timed(1e9, args.steps)
        print(json.dumps({"quick": True, "workload": w, "steps": n, "ms_per_step": ms / n,
                          "value": NX * NY * n / (ms / 1e3)}))
        s.close()
        return 0
    if w == "mlp-train":
        import numpy as np
        rng = np.random.default_rng(0)
        X = rng.normal(0, 1, (65536, gdf.NFEAT)).astype(np.float32)
        y = (X[:, :8].sum(1) > 1.0).astype(np.float32)
        m = gdf.Mlp(0)
        t0 = time.perf_counter()
        loss = m.train(X, y, epochs=1, batch=2048, lr=1e-3)
        print(json.dumps({"quick": True, "workload": w, "loss": float(loss[0]),
                          "seconds": time.perf_counter() - t0}))
        return 0
    from gdf.indicator import WEIGHTS, load_net
    net, lo, hi = load_net(WEIGHTS)
    if w == "blast-learned":
        cfg, tend = gdf.problem_config(gdf.PROB_BLAST, 512, 512)
        cfg.detector = gdf.DETECT_LEARNED
        s = gdf.Solver(cfg)
        s.set_indicator(net, lo, hi)
        s.upload(*gdf.init_data(cfg, gdf.PROB_BLAST))
        s.prepare()
        if args.warmup:
            s.advance_timed(tend, args.warmup)
        _, n, ms = s.advance_timed(tend, args.steps)
        print(json.dumps({"quick": True, "workload": w, "steps": n, "ms_per_step": ms / n,
                          "value": 512 * 512 * n / (ms / 1e3)}))
        s.close()
        return 0
    # ensemble-small
    items = []
    for i, (prob, side) in enumerate([(gdf.PROB_ORSZAG_TANG, 64), (gdf.PROB_ROTOR, 96), (gdf.PROB_BLAST, 128),
                                      (gdf.PROB_ROTOR, 160), (gdf.PROB_BLAST, 64), (gdf.PROB_ORSZAG_TANG, 128),
                                      (gdf.PROB_ROTOR, 64), (gdf.PROB_BLAST, 96)]):
        c, te = gdf.problem_config(prob, side, side)
        c.flux_type = gdf.FLUX_HLLD
        c.faceb_limiter = 1
        c.detector = gdf.DETECT_LEARNED
        c.kxrcf_ck = 1.0
        items.append((c, prob, te))
    e = gdf.Ensemble([c for c, _, _ in items])
    e.set_indicator(net, lo, hi)
    for i, (c, prob, te) in enumerate(items):
        e.upload(i, *gdf.init_data(c, prob))
    e.prepare()
    for i, (_, _, te) in enumerate(items):
        e.set_time(i, 0.0, te)
    if args.warmup:
        e.advance(args.warmup)
    cu, act, ms = e.advance(args.steps)
    print(json.dumps({"quick": True, "workload": w, "steps": args.steps, "ms_per_step": ms / args.steps,
                      "value": cu / (ms / 1e3), "tiles": e.tiles()}))
    e.close()
    return 0


def run_ours(args):
    world, rank, local = dist_env()
    import numpy as np
    import gdf
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    gdf.set_device(local)
    cfg, uh, bx, by = make_state(gdf)
    s = gdf.Solver(cfg)
    s.upload(uh, bx, by)
    s.prepare()
    s.advance_timed(1e9, max(3, args.warmup))       # warm-up (also captures the step graph)
    if dist:
        dist.barrier()
    clk = ClockSampler(local)
    clk.start()
    time.sleep(0.05)
    l0 = s.kernel_launches()
    h0 = time.perf_counter()
    _, taken, ms = s.advance_timed(1e9, args.steps)   # returns after the device finished
    clk.mark(h0, time.perf_counter())
    launches = s.kernel_launches() - l0
    clocks = clk.stop()
    ms_max = reduce_max_ms(ms, dist, f"cuda:{local}")
    value = job_value(world, args.steps, ms_max)

    # per-kernel timing (events around every launch) for the roofline
    prof = s.profile(2)
    dom = max((k for k in prof if k in ALG_BYTES_PER_CELL), key=lambda k: prof[k][0] * prof[k][1])
    dom_ms, dom_per_step = prof[dom]
    # with a detector the limiter runs in two passes: the first reads every
    # cell and writes the ungated ones, the second takes the gated cells (the
    # sticky KXRCF flags)
    flagged = int((s.trouble() != 0).sum())
    ncell = NX * NY
    if dom == "limit_tvb":
        alg_bytes = ALG_BYTES_PER_CELL["limit_tvb"] * flagged
    elif dom == "limit":
        alg_bytes = 416 * ncell + (416 + 4) * (ncell - flagged) + 4 * flagged
        if not cfg.faceb_limiter:
            alg_bytes += (ALG_BYTES_LIMIT_FUSED - ALG_BYTES_PER_CELL["limit"]) * (ncell - flagged)
    else:
        alg_bytes = ALG_BYTES_PER_CELL[dom] * ncell
    peak, peak_kind = read_peaks()
    achieved = alg_bytes / (dom_ms / 1e3) / 1e9
    traffic = None
    tp = os.path.join(REPO, "profiles", "traffic_rotor512.json")
    if os.path.exists(tp):
        try:
            traffic = json.load(open(tp)).get(dom)
        except Exception:
            traffic = None

    # end to end through the public API with host buffers (pinned)
    import torch
    pin = lambda a: torch.from_numpy(a).pin_memory().numpy()   # noqa: E731
    huh, hbx, hby = pin(uh), pin(bx), pin(by)
    s.upload(huh, hbx, hby)
    s.prepare()
    huh2, hbx2, hby2 = s.download()
    huh, hbx, hby = pin(huh2), pin(hbx2), pin(hby2)
    e2e_steps = max(2, min(args.steps, 10))
    t = 0.0
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        s.upload(huh, hbx, hby)
        s.t = t
        t, _, _ = s.step(1e9, flags=False)
        s.download_into(huh, hbx, hby, live_only=True)
    e2e_el = time.perf_counter() - t0
    e2e = world * NX * NY * e2e_steps / e2e_el
    io_bytes = huh.nbytes + hbx.nbytes + hby.nbytes
    # gdf_upload moves the 52 live slot planes of uh (the 28 dead ones are
    # checked to be zero on the host and stay zero on the device)
    h2d_bytes = huh.nbytes * 52 // 80 + hbx.nbytes + hby.nbytes

    # the opt-in FMA build on the same workload, for comparison
    fma = None
    if not args.no_fma:
        f = gdf.Solver(cfg, exact=False)
        f.upload(uh, bx, by)
        f.prepare()
        f.advance_timed(1e9, 3)
        _, _, fms = f.advance_timed(1e9, args.steps)
        fma = {"value": NX * NY * args.steps / (fms / 1e3), "unit": UNIT, "ms_per_step": fms / args.steps,
               "build": "libgdf_b200_fma.so (FMA contraction; not tie-exact)"}
        f.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(gdf, args.cpu_steps)

    learned = ens = None
    if not args.no_extra and rank == 0 and world == 1:
        try:
            learned = learned_blast(gdf, args.steps)
        except Exception as e:   # reported, not fatal: the headline line still prints
            learned = {"error": str(e)}
        try:
            ens = ensemble_bench(gdf, args.steps)
        except Exception as e:
            ens = {"error": str(e)}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "grid": [NX, NY], "problem": "rotor", "method": "plain",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": "inputs larger than L2 (uh alone is 168 MB per copy; 126 MB L2)",
                       "timing": "CUDA events on the library stream around graph replays"},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "alg_bytes_per_launch": alg_bytes, "ms_per_launch": dom_ms,
                         "launches_per_step": dom_per_step, "flagged_cells": flagged},
            "kernels_ms_per_launch": {k: v[0] for k, v in prof.items() if v[1]},
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(h2d_bytes),
                    "d2h_bytes_per_step": int(h2d_bytes), "steps": e2e_steps,
                    "calls": "gdf_upload, gdf_step, gdf_download_live per step (pinned host arrays)"},
            "cpu_baseline": cpu,
            "fma_build": fma,
            "learned_indicator": learned,
            "ensemble": ens,
            "build": "libgdf_b200.so (no FMA contraction: value-exact with the reference arithmetic)",
            "clocks": clocks,
            "steps_taken": taken,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    s.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--no-fma", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the learned-indicator and ensemble runs")
    ap.add_argument("--quick", action="store_true", help="timed steps only (for profiler captures)")
    ap.add_argument("--fma", action="store_true", help="with --quick: run the FMA build")
    ap.add_argument("--workload", default="rotor", choices=["rotor", "blast-learned", "ensemble-small", "mlp-train"],
                    help="with --quick: what to run")
    args = ap.parse_args()
    if args.quick:
        return run_quick(args)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
