"""bench.py's multi-GPU path is replicas only: each rank advances its own
copy of the workload and the job time is the max over ranks. The rank
logic runs here on CPU with the gloo backend, world size 2."""
import json
import os
import subprocess
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ms = 10.0 + 5.0 * rank          # rank 1 is the slow one
    m = bench.reduce_max_ms(ms, dist, "cpu")
    v = bench.job_value(world, bench.NX * bench.NY, 4, m)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, m, v))


def test_max_over_ranks_and_job_value():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    import bench
    for rank, m, v in res:
        assert m == 15.0
        assert v == pytest.approx(2 * bench.NX * bench.NY * 4 / 0.015)


def test_reference_arm_nonzero_rank_exits_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""


def test_cpu_sample_band_is_a_slice_of_the_blast_grid():
    """The reference arm's band has the blast grid's cell size, its cells
    sit on the blast grid's cell centres, and its share of cells inside the
    initial blast disc is close to the whole grid's."""
    import numpy as np
    import bench
    from gdf._abi import PROB_BLAST, problem_config
    cfg, _ = problem_config(PROB_BLAST, bench.NX, bench.NY)
    b = bench.band_config(cfg)
    h = (cfg.yb - cfg.ya) / cfg.ny
    assert (b.nx, b.ny) == (cfg.nx, bench.BAND)
    assert abs((b.yb - b.ya) / b.ny - h) < 1e-15 and (b.xa, b.xb) == (cfg.xa, cfg.xb)
    yc_band = b.ya + (np.arange(b.ny) + 0.5) * h
    yc_full = cfg.ya + (np.arange(cfg.ny) + 0.5) * h
    assert np.allclose(yc_band, yc_full[bench.BAND_Y0:bench.BAND_Y0 + bench.BAND], atol=1e-14)
    xc = cfg.xa + (np.arange(cfg.nx) + 0.5) * h

    def share(yc):
        X, Y = np.meshgrid(xc, yc)
        return float(((X * X + Y * Y) < 0.01).mean())
    s_band, s_full = share(yc_band), share(yc_full)
    assert abs(s_band - s_full) < 0.005, (s_band, s_full)


def test_single_rank_reduce_is_identity():
    import bench
    assert bench.reduce_max_ms(3.5, None, "cpu") == 3.5


def test_clock_sampler_counts_only_the_timed_window(monkeypatch):
    """Clock samples outside the host times that bracket the timed region
    are left out; the clock-event reason bits decode to their names; with no
    sample inside a short window the nearest one stands in."""
    import bench
    c = bench.ClockSampler(0)
    c.samples = [(1.0, 1100.0, 1965.0, 0x1), (2.0, 1965.0, 1965.0, 0x4), (2.5, 1950.0, 1965.0, 0x4 | 0x40),
                 (9.0, 900.0, 1965.0, 0x8)]
    c.mark(1.5, 3.0)
    r = c.stop()
    assert r["samples"] == 2 and r["sm_mhz"] == 1957.5 and r["sm_max_mhz"] == 1965.0
    assert r["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]
    c = bench.ClockSampler(0)
    c.samples = [(1.0, 1000.0, 1965.0, 0), (5.0, 1965.0, 1965.0, 0)]
    c.mark(4.5, 4.6)
    r = c.stop()
    assert r["samples"] == 1 and r["sm_mhz"] == 1965.0 and r["reasons"] == []
    monkeypatch.setenv("CUDA_VISIBLE_DEVICES", "GPU-1234,3")
    calls = []

    class FakeNvml:
        @staticmethod
        def nvmlDeviceGetHandleByUUID(u):
            calls.append(("uuid", u))

        @staticmethod
        def nvmlDeviceGetHandleByIndex(i):
            calls.append(("index", i))
    monkeypatch.setitem(sys.modules, "pynvml", FakeNvml)
    bench.nvml_index(0)
    bench.nvml_index(1)
    bench.nvml_index(2)
    assert calls == [("uuid", "GPU-1234"), ("index", 3), ("index", 2)]
