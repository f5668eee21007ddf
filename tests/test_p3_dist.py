"""The k = 3 variant's block decomposition (gdf/p3_dist.py), the
reference's MPI layout (MPI_BalsaraP3/main.f90:8-11, set_bc :1574-1867).

On the CPU: the ghost layers a decomposition fills, between blocks in one
process and between gloo ranks (world size 2), equal the ghost layers
set_bc gives the undivided grid (the oracle's set_bc on random data), for
periodic and outflow edges and for a periodic axis of two blocks, where
each rank is the other's neighbour on both sides.
On the GPU: a 2 x 2 decomposed run equals the single-block run value for
value.
"""
import datetime
import os
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import gdf
from gdf import p3
from gdf.p3 import p3_problem_config
from gdf.p3_dist import BlockGrid, DistTransport, LocalTransport, P3Decomposed

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _global_case(problem, nx, ny, seed=0):
    """Random cells and faces, the oracle's set_bc applied: the reference
    ghost layers. Returns the config, the (84, NY+2, NX+2) slot planes and
    the face arrays before and after."""
    from oracle import OracleP3
    cfg, _ = p3_problem_config(problem, nx, ny)
    rng = np.random.default_rng(seed)
    uh, bx, by = p3.p3_new_state(nx, ny)
    live = p3.p3_live_mask()
    uh[live] = rng.normal(size=uh[live].shape)
    bx[:] = rng.normal(size=bx.shape)
    by[:] = rng.normal(size=by.shape)
    ref = [a.copy() for a in (uh, bx, by)]
    OracleP3(cfg).set_bc(*ref)
    return cfg, uh[live], bx, by, ref[0][live], ref[1], ref[2]


def _block_views(grid, cells, bx, by, b):
    bi, bj = b
    x0, y0 = bi * grid.nxb, bj * grid.nyb
    c = torch.from_numpy(np.ascontiguousarray(cells[:, y0:y0 + grid.nyb + 2, x0:x0 + grid.nxb + 2]))
    fx = torch.from_numpy(np.ascontiguousarray(bx[:, y0:y0 + grid.nyb + 2, x0:x0 + grid.nxb + 1]))
    fy = torch.from_numpy(np.ascontiguousarray(by[:, y0:y0 + grid.nyb + 1, x0:x0 + grid.nxb + 2]))
    return c, fx, fy


def _check_block(grid, b, c, fx, fy, rc, rbx, rby):
    bi, bj = b
    x0, y0 = bi * grid.nxb, bj * grid.nyb
    assert np.array_equal(c.numpy(), rc[:, y0:y0 + grid.nyb + 2, x0:x0 + grid.nxb + 2]), b
    assert np.array_equal(fx.numpy(), rbx[:, y0:y0 + grid.nyb + 2, x0:x0 + grid.nxb + 1]), b
    assert np.array_equal(fy.numpy(), rby[:, y0:y0 + grid.nyb + 1, x0:x0 + grid.nxb + 2]), b


@pytest.mark.parametrize("problem,px,py", [(gdf.PROB_ORSZAG_TANG, 2, 2), (gdf.PROB_CLOUD_SHOCK, 2, 2),
                                           (gdf.PROB_ORSZAG_TANG, 3, 1), (gdf.PROB_CLOUD_SHOCK, 1, 3),
                                           (gdf.PROB_ORSZAG_TANG, 1, 1)])
def test_local_ghost_fill_equals_set_bc(problem, px, py):
    cfg, cells, bx, by, rc, rbx, rby = _global_case(problem, 12, 12)
    grid = BlockGrid(cfg, px, py)
    views = {b: _block_views(grid, cells, bx, by, b) for b in grid.blocks()}
    tr = LocalTransport(grid)
    tr.fill({b: v[0] for b, v in views.items()}, "cells")
    tr.fill({b: (v[1], v[2]) for b, v in views.items()}, "faces")
    for b, (c, fx, fy) in views.items():
        _check_block(grid, b, c, fx, fy, rc, rbx, rby)


def test_blocks_split_and_join_and_keep_the_grid_spacing():
    cfg, _ = p3_problem_config(gdf.PROB_ORSZAG_TANG, 12, 8)
    grid = BlockGrid(cfg, 3, 2)
    bc = grid.block_config()
    assert (bc.nx, bc.ny, bc.nx_global, bc.ny_global) == (4, 4, 12, 8)
    assert (bc.xa, bc.xb) == (cfg.xa, cfg.xb)
    uh, bx, by = p3.p3_new_state(12, 8)
    rng = np.random.default_rng(1)
    uh[p3.p3_live_mask()] = rng.normal(size=uh[p3.p3_live_mask()].shape)
    bx[:, 1:-1, :] = rng.normal(size=bx[:, 1:-1, :].shape)
    by[:, :, 1:-1] = rng.normal(size=by[:, :, 1:-1].shape)
    uh[:, :, 0, :] = uh[:, :, -1, :] = uh[:, :, :, 0] = uh[:, :, :, -1] = 0
    parts = {b: grid.split(uh, bx, by, *b) for b in grid.blocks()}
    ju, jx, jy = grid.join(parts)
    assert np.array_equal(ju, uh) and np.array_equal(jx, bx) and np.array_equal(jy, by)
    with pytest.raises(ValueError):
        BlockGrid(cfg, 5, 2)


def _dist_worker(rank, world, port, problem, px, py, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, os.path.join(REPO, "freljord-cfd-arsenal_b200"))
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        cfg, cells, bx, by, rc, rbx, rby = _global_case(problem, 12, 10, seed=7)
        grid = BlockGrid(cfg, px, py)
        tr = DistTransport(grid, dist)
        b = grid.block_of(rank)
        c, fx, fy = _block_views(grid, cells, bx, by, b)
        tr.fill({b: c}, "cells")
        tr.fill({b: (fx, fy)}, "faces")
        _check_block(grid, b, c, fx, fy, rc, rbx, rby)
        ax, ay = tr.max_speeds([(1.0 + rank, 5.0 - rank)])
        assert (ax, ay) == (float(world), 5.0)
        dist.barrier()
        q.put((rank, "ok"))
    except Exception as e:   # reported to the parent
        q.put((rank, repr(e)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("problem,px,py", [(gdf.PROB_ORSZAG_TANG, 2, 1), (gdf.PROB_CLOUD_SHOCK, 2, 1),
                                           (gdf.PROB_ORSZAG_TANG, 1, 2)])
def test_gloo_ranks_fill_the_ghosts_of_set_bc(problem, px, py):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29700 + (os.getpid() + 31 * px + 7 * problem) % 1000
    procs = [ctx.Process(target=_dist_worker, args=(r, 2, port, problem, px, py, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert res == [(0, "ok"), (1, "ok")], res
    assert all(p.exitcode == 0 for p in procs)


@pytest.mark.gpu
@pytest.mark.parametrize("problem,nx,ny,px,py", [(gdf.PROB_ORSZAG_TANG, 32, 32, 2, 2),
                                                 (gdf.PROB_CLOUD_SHOCK, 40, 20, 2, 2),
                                                 (gdf.PROB_ROTOR, 24, 24, 3, 1)])
def test_decomposed_run_equals_single_block(problem, nx, ny, px, py):
    cfg, tend = p3_problem_config(problem, nx, ny)
    state = p3.p3_init_data(cfg, problem)
    one = p3.P3Solver(cfg)
    one.upload(*state)
    one.prepare()
    grid = BlockGrid(cfg, px, py)
    dec = P3Decomposed(grid, LocalTransport(grid))
    dec.upload(*state)
    dec.prepare()
    for k in range(3):
        t1, dt1 = one.step(tend)
        t2, dt2 = dec.step(tend)
        assert (t1, dt1) == (t2, dt2), k
        u1, x1, y1 = one.download()
        u2, x2, y2 = dec.download()
        assert np.array_equal(u1[:, :, 1:-1, 1:-1], u2[:, :, 1:-1, 1:-1]), k
        assert np.array_equal(x1[:, 1:-1, :], x2[:, 1:-1, :]) and np.array_equal(y1[:, :, 1:-1], y2[:, :, 1:-1]), k
