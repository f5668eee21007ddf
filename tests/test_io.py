"""The reference's output files (save_solution.f90, RK3.f90 frames,
save_XY.f90), its L2 error (calculate_L2error.f90), the binary checkpoint,
and the main.f90 driver."""
import math
import os

import numpy as np
import pytest

import gdf


def small_state(problem=gdf.PROB_ORSZAG_TANG, nx=6, ny=4):
    cfg, tend = gdf.problem_config(problem, nx, ny)
    uh, bx, by = gdf.init_data(cfg, problem)
    return cfg, tend, uh, bx, by


def test_save_solution_layout(tmp_path):
    cfg, _, uh, _, _ = small_state()
    uh[5, 6] = np.linspace(-1, 1, uh[5, 6].size).reshape(uh[5, 6].shape)   # a Bx cubic mode
    gdf.save_solution(cfg, uh, str(tmp_path))
    for n in range(8):
        q = np.loadtxt(tmp_path / f"Q{n + 1}.txt")
        assert q.shape == (10 * cfg.ny * cfg.nx,)
        # d, then j, then i; 17 significant digits read back exactly
        assert np.array_equal(q, uh[n, :, 1:-1, 1:-1].ravel())


def test_save_frames_append(tmp_path):
    cfg, _, uh, _, _ = small_state()
    gdf.save_frame(cfg, uh, 0.0, str(tmp_path), reset=True)
    gdf.save_frame(cfg, 2 * uh, 0.25, str(tmp_path))
    t = np.loadtxt(tmp_path / "T.txt")
    assert np.array_equal(t, [0.0, 0.25])
    q = np.loadtxt(tmp_path / "Q5flash.txt").reshape(2, -1)
    assert np.array_equal(q[0], uh[4, :, 1:-1, 1:-1].ravel()) and np.array_equal(q[1], 2 * uh[4, :, 1:-1, 1:-1].ravel())
    gdf.save_frame(cfg, uh, 0.0, str(tmp_path), reset=True)
    assert np.loadtxt(tmp_path / "T.txt").size == 1


def test_save_xy(tmp_path):
    cfg, _, _, _, _ = small_state(nx=5, ny=3)
    gdf.save_xy(cfg, str(tmp_path))
    lam = np.loadtxt(tmp_path / "lambda.txt")
    w = np.loadtxt(tmp_path / "weight.txt")
    assert lam.size == 5 and abs(w.sum() - 2.0) < 1e-14 and abs(lam.sum()) < 1e-15
    hx = (cfg.xb - cfg.xa) / cfg.nx
    xc = cfg.xa + (np.arange(1, cfg.nx + 1) - 0.5) * hx
    assert np.allclose(np.loadtxt(tmp_path / "Xc.txt"), (xc[:, None] + 0.5 * hx * lam[None, :]).ravel(), rtol=0,
                       atol=1e-14)
    assert np.loadtxt(tmp_path / "Yc.txt").size == cfg.ny * 5


def vortex_exact(x, y):
    r2 = x * x + y * y
    e = np.exp(0.5 * (1 - r2))
    p = 1 - r2 / (8 * math.pi ** 2) * np.exp(1 - r2)
    u = 1 - y * e / (2 * math.pi)
    v = 1 + x * e / (2 * math.pi)
    b1 = -y * e / (2 * math.pi)
    b2 = x * e / (2 * math.pi)
    E = p / (5.0 / 3.0 - 1) + 0.5 * (u * u + v * v) + 0.5 * (b1 * b1 + b2 * b2)
    z = np.zeros_like(x)
    return [np.ones_like(x), u, v, z, E, b1, b2, z]


def l2_numpy(cfg, uh, t20):
    g = np.array([-0.9061798459386639927976269, -0.5384693101056830910363144, 0,
                  0.5384693101056830910363144, 0.9061798459386639927976269])
    w = np.array([0.2369268850561890875142640, 0.4786286704993664680412915, 0.5688888888888888888888889,
                  0.4786286704993664680412915, 0.2369268850561890875142640])
    li, lj = np.meshgrid(g, g, indexing="ij")
    basis = [np.ones_like(li), li, lj, li ** 2 - 1 / 3, li * lj, lj ** 2 - 1 / 3, li ** 3 - 0.6 * li,
             (li ** 2 - 1 / 3) * lj, li * (lj ** 2 - 1 / 3), lj ** 3 - 0.6 * lj]
    hx, hy = (cfg.xb - cfg.xa) / cfg.nx, (cfg.yb - cfg.ya) / cfg.ny
    acc = np.zeros(8)
    for j in range(1, cfg.ny + 1):
        for i in range(1, cfg.nx + 1):
            x = cfg.xa + (i - 0.5) * hx + 0.5 * hx * li - t20
            y = cfg.ya + (j - 0.5) * hy + 0.5 * hy * lj - t20
            ex = vortex_exact(x, y)
            for n in range(8):
                num = sum(uh[n, d, j, i] * basis[d] for d in range(10))
                acc[n] += np.sum(np.outer(w, w) * (num - ex[n]) ** 2)
    return np.sqrt(acc * 0.25 * hx * hy)


def test_l2_error_matches_numpy_and_converges():
    errs = []
    for n in (8, 16, 32):
        cfg, _ = gdf.problem_config(gdf.PROB_VORTEX, n, n)
        uh, _, _ = gdf.init_data(cfg, gdf.PROB_VORTEX)
        L2 = gdf.l2_error(cfg, uh, 0.0)
        if n == 8:
            ref = l2_numpy(cfg, uh, 0.0)
            live = ref > 1e-300
            assert np.allclose(L2[live], ref[live], rtol=1e-10, atol=0)
        errs.append(L2[0] + L2[1])
    # the P2 L2 projection of the smooth vortex: third order
    assert math.log2(errs[1] / errs[2]) > 2.7


@pytest.mark.gpu
def test_checkpoint_restart_is_value_exact(tmp_path):
    cfg, tend, uh, bx, by = small_state(gdf.PROB_ROTOR, 24, 24)
    a = gdf.Solver(cfg)
    a.upload(uh, bx, by)
    a.prepare()
    a.advance(tend, 4)
    path = str(tmp_path / "rotor.ckpt")
    a.checkpoint(path)
    a.advance(tend, 5)
    b = gdf.Solver(cfg)
    b.restore(path)
    assert b.t > 0
    b.advance(tend, 5)
    for x, y in zip(a.download(), b.download()):
        assert np.array_equal(x, y)
    assert a.time()[0] == b.time()[0]
    assert np.array_equal(a.trouble(), b.trouble()) and a.trouble().any()
    other, _ = gdf.problem_config(gdf.PROB_ROTOR, 24, 20)
    c = gdf.Solver(other)
    with pytest.raises(gdf.GdfError):
        c.restore(path)


@pytest.mark.gpu
def test_main_driver_writes_the_reference_files(tmp_path):
    from gdf.run import run
    out = str(tmp_path / "ot")
    t, steps, L2 = run(gdf.PROB_ORSZAG_TANG, 16, 16, out, tend=0.05, flash=True, frame_max=4)
    assert t == 0.05 and steps > 1 and L2.shape == (8,)
    frames = np.loadtxt(os.path.join(out, "T.txt"))
    assert frames[0] == 0.0 and frames[-1] == 0.05 and 3 <= frames.size <= 6
    for name in ["Q1.txt", "Q8.txt", "Xc.txt", "Yc.txt", "lambda.txt", "weight.txt", "Q3flash.txt"]:
        assert os.path.exists(os.path.join(out, name))
    q1 = np.loadtxt(os.path.join(out, "Q1flash.txt")).reshape(frames.size, -1)
    assert np.array_equal(q1[-1], np.loadtxt(os.path.join(out, "Q1.txt")))


@pytest.mark.gpu
def test_download_live_writes_only_live_planes():
    cfg, tend, uh, bx, by = small_state(gdf.PROB_ROTOR, 20, 16)
    s = gdf.Solver(cfg)
    s.upload(uh, bx, by)
    s.prepare()
    s.advance(tend, 2)
    full = s.download()
    marked = np.full_like(uh, 7.0)
    b1, b2 = np.zeros_like(bx), np.zeros_like(by)
    s.download_into(marked, b1, b2, live_only=True)
    live = np.zeros((8, 10), bool)
    live[:, :6] = True
    live[5, [6, 8]] = True
    live[6, [7, 9]] = True
    assert np.array_equal(marked[live], full[0][live])
    assert np.all(marked[~live] == 7.0)
    assert np.array_equal(b1, full[1]) and np.array_equal(b2, full[2])


@pytest.mark.gpu
def test_driver_checkpoint_restart_continues_value_exact(tmp_path):
    from gdf.run import run
    full, part = str(tmp_path / "full"), str(tmp_path / "part")
    ckpt = str(tmp_path / "r.ckpt")
    t5, n5, _ = run(gdf.PROB_ROTOR, 24, 20, full, tend=1.0, max_steps=5)
    t3, n3, L2 = run(gdf.PROB_ROTOR, 24, 20, part, tend=1.0, max_steps=3, checkpoint=ckpt, save=False)
    assert (n5, n3) == (5, 3) and L2 is None and not os.path.exists(os.path.join(part, "Q1.txt"))
    t, n, _ = run(gdf.PROB_ROTOR, 24, 20, part, tend=1.0, max_steps=2, restart=ckpt)
    assert n == 2 and t == t5 and t3 < t5
    for q in ("Q1.txt", "Q6.txt", "Q7.txt"):
        assert np.array_equal(np.loadtxt(os.path.join(full, q)), np.loadtxt(os.path.join(part, q)))
