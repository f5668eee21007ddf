"""The ensemble (gdf_ens_*): independent problems of different sizes and
settings advanced by one persistent kernel per RK stage must each follow,
value for value, the trajectory a single-problem handle computes for them;
with per-instance dt, per-instance end times, any tile shape, the learned
indicator, and across the autotuner's trials."""
import numpy as np
import pytest

import gdf

pytestmark = pytest.mark.gpu


def mixed_instances():
    """(config, problem, params, tend) of small instances with different
    sizes, domains, fluxes, detectors and face-B limiting."""
    out = []
    for prob, nx, ny, edit in [
        (gdf.PROB_ORSZAG_TANG, 24, 20, None),                       # HLL, all-cells limiter
        (gdf.PROB_ROTOR, 32, 32, None),                             # HLLD, KXRCF + pp
        (gdf.PROB_BLAST, 20, 28, None),                             # HLLD, KXRCF, face-B limiter
        (gdf.PROB_CLOUD_SHOCK, 24, 12, lambda c: setattr(c, "flux_type", gdf.FLUX_LF)),
        (gdf.PROB_VORTEX, 16, 16, None),
        (gdf.PROB_ROTOR, 40, 24, lambda c: setattr(c, "flux_type", gdf.FLUX_HLLC)),
    ]:
        cfg, tend = gdf.problem_config(prob, nx, ny)
        if edit:
            edit(cfg)
        out.append((cfg, prob, None, tend))
    return out


def run_single(cfg, prob, params, tend, steps, net=None, lohi=(0.5, 0.5)):
    uh, bx, by = gdf.init_data(cfg, prob, params)
    s = gdf.Solver(cfg)
    if net is not None:
        s.set_indicator(net, *lohi)
    s.upload(uh, bx, by)
    s.prepare()
    s.advance(tend, steps)
    return s.download(), s.time()[0]


def make_ensemble(insts, net=None, lohi=(0.5, 0.5), tends=None):
    e = gdf.Ensemble([c for c, _, _, _ in insts])
    if net is not None:
        e.set_indicator(net, *lohi)
    for i, (cfg, prob, params, _) in enumerate(insts):
        e.upload(i, *gdf.init_data(cfg, prob, params))
    e.prepare()
    for i, (_, _, _, tend) in enumerate(insts):
        e.set_time(i, 0.0, tends[i] if tends else tend)
    return e


def same(a, b):
    return all(np.array_equal(x, y) for x, y in zip(a, b))


@pytest.mark.parametrize("mode", [0, 1], ids=["persistent", "per-phase"])
def test_ensemble_matches_single_problem_handles(mode):
    insts = mixed_instances()
    # the vortex instance stops after about two steps: its end time is short
    tends = [1e9] * len(insts)
    tends[4] = 0.07
    e = make_ensemble(insts, tends=tends)
    e.set_mode(mode)
    steps = 5
    cu, active, ms = e.advance(steps)
    assert ms > 0
    total = 0
    for i, (cfg, prob, params, _) in enumerate(insts):
        ref, t_ref = run_single(cfg, prob, params, tends[i], steps)
        got = e.download(i)
        assert same(got, ref), f"instance {i} differs"
        t, _, n = e.time(i)
        assert t == t_ref
        total += n * cfg.nx * cfg.ny
    assert e.time(4)[2] < steps and e.time(0)[2] == steps
    assert cu == total and active == len(insts) - 1


def test_tile_shapes_and_modes_give_identical_results():
    insts = mixed_instances()[:3]
    res = []
    for mode, tiles in [(0, (0, 1, 1)), (0, (1, 4, 2)), (0, (2, 2, 4)), (1, (0, 1, 1)), (1, (0, 4, 2))]:
        e = make_ensemble(insts)
        e.set_mode(mode)
        e.set_tiles(*tiles)
        e.advance(3)
        res.append([e.download(i) for i in range(len(insts))])
        e.close()
    for r in res[1:]:
        assert all(same(a, b) for a, b in zip(r, res[0]))


def test_autotuner_keeps_the_trajectory():
    insts = mixed_instances()[:4]
    a = make_ensemble(insts)
    ms = a.tune(1)
    assert ms.shape == (gdf.ENS_TUNE_CANDIDATES,) and (ms[:36] > 0).any() and (ms[36:] > 0).all()
    tl = a.tiles()
    assert tl["grid"] > 0 and tl["face_per_thread"] in (1, 2, 4) and tl["mode"] in (0, 1)
    a.advance(3)
    b = make_ensemble(insts)
    b.advance(3)
    for i in range(len(insts)):
        assert same(a.download(i), b.download(i))
        assert a.time(i) == b.time(i)


@pytest.mark.parametrize("mode", [0, 1], ids=["persistent", "per-phase"])
def test_learned_ensemble_matches_single_problem_handles(mode):
    net = gdf.Mlp(11)
    insts = []
    for cfg, prob, params, tend in mixed_instances()[:4]:
        cfg.detector = gdf.DETECT_LEARNED
        cfg.kxrcf_ck = 1.0
        insts.append((cfg, prob, params, tend))
    lohi = (0.3, 0.7)
    e = make_ensemble(insts, net, lohi)
    e.set_mode(mode)
    e.advance(3)
    for i, (cfg, prob, params, tend) in enumerate(insts):
        ref, t_ref = run_single(cfg, prob, params, tend, 3, net, lohi)
        assert same(e.download(i), ref), f"instance {i} differs"


def test_ensemble_workload_configs():
    cfgs = gdf.ensemble_configs(64, seed=0)
    sides = {c.nx for c, _, _, _ in cfgs}
    assert len(cfgs) == 64 and sides <= set(range(64, 513, 32)) and len(sides) > 8
    assert {p for _, p, _, _ in cfgs} == {gdf.PROB_ORSZAG_TANG, gdf.PROB_ROTOR, gdf.PROB_BLAST}
    assert all(c.flux_type == gdf.FLUX_HLLD and c.detector == gdf.DETECT_LEARNED for c, _, _, _ in cfgs)


def test_ensemble_errors():
    insts = mixed_instances()[:2]
    e = gdf.Ensemble([c for c, _, _, _ in insts])
    with pytest.raises(gdf.GdfError):
        e.advance(1)                        # nothing uploaded
    with pytest.raises(gdf.GdfError):
        e.set_indicator(gdf.Mlp(0))         # detectors are not learned
    with pytest.raises(gdf.GdfError):
        e.set_tiles(0, 0, 1)
    with pytest.raises(gdf.GdfError):
        e.set_mode(2)
    cfg = insts[0][0].copy()
    cfg.nx = 1
    with pytest.raises(gdf.GdfError):
        gdf.Ensemble([insts[1][0], cfg])


def test_bounded_barrier_reports_a_missing_block_and_device_stays_usable():
    """The persistent mode's grid barrier waits with a time limit: a block
    that never arrives (a flag nothing sets) makes the others give up after
    the limit and report it; nothing faults, and the device keeps working."""
    import time
    assert gdf.ens_barrier_selftest(16, -1, 2_000_000_000) is False
    t0 = time.time()
    assert gdf.ens_barrier_selftest(16, 5, 50_000_000) is True
    assert time.time() - t0 < 30
    insts = mixed_instances()[:2]
    e = make_ensemble(insts)
    e.set_mode(0)
    e.advance(2)
    for i, (cfg, prob, params, tend) in enumerate(insts):
        ref, _ = run_single(cfg, prob, params, tend, 2)
        assert same(e.download(i), ref)
