"""The cylindrical variant's CUDA path against the oracle, value for value.

Every entry point of include/gdf_cy.h that computes is compared with the CPU
restatement of MHD_GDF_cy3D_0421/ on the same inputs: Lh + LhEz (du, dBr,
dBz on every cell and face), the limiter (TVB_Limiter_P2 +
div_free_Balsara), dt, whole RK3 steps (interior cells and all faces; the
ghost layers are refreshed by set_bc before every use and carry no state),
the graph-replayed advance and the diagnostics, over the problems, boundary
codes (1-5 in r, 1, 2, 4 in z), fluxes (central, LF, HLL) and plane counts
(Lphi 1, 2, 4). The product build has no FMA contraction, so the
comparisons are exact (==). Two tolerances, each stated where it is used:
the manufactured-solution source (Source.f90) evaluates sin and cos with
CUDA's device functions, which differ from the host's in the last bits
(1e-12 relative on Lh, 1e-10 after steps), and totaldiv sums per-cell terms
in a different grouping (1e-12 relative).
"""
import numpy as np
import pytest

from gdf import cy
from gdf.cy import cy_problem_config
from oracle import OracleCy

pytestmark = pytest.mark.gpu


def _interior(a):
    return a[:, :, :, 1:-1, 1:-1]


def _state(problem, nr, nz, lphi, flux=None, steps=0, **over):
    cfg, tend = cy_problem_config(problem, nr, nz, lphi)
    if flux is not None:
        cfg.flux_type = flux
    for k, v in over.items():
        setattr(cfg, k, v)
    o = OracleCy(cfg)
    uh, br, bz = o.init_data(problem)
    o.limit(uh, br, bz)
    t = 0.0
    for _ in range(steps):
        t, _ = o.step(uh, br, bz, t, tend if tend > 0 else 1.0)
    return cfg, tend, o, uh, br, bz, t


@pytest.mark.parametrize("problem,lphi,flux", [
    (cy.CY_ORSZAG_TANG, 1, cy.CY_FLUX_HLL), (cy.CY_ORSZAG_TANG, 1, cy.CY_FLUX_LF),
    (cy.CY_ORSZAG_TANG, 1, cy.CY_FLUX_CENTRAL), (cy.CY_ORSZAG_TANG2, 2, cy.CY_FLUX_HLL),
    (cy.CY_ORSZAG_TANG2, 4, cy.CY_FLUX_LF), (cy.CY_EXPLOSION, 1, cy.CY_FLUX_HLL),
    (cy.CY_ROTOR, 1, cy.CY_FLUX_HLL), (cy.CY_JET, 2, cy.CY_FLUX_HLL), (cy.CY_DIV_TEST, 2, cy.CY_FLUX_HLL)])
def test_lh_matches_oracle(problem, lphi, flux):
    cfg, tend, o, uh, br, bz, t = _state(problem, 20, 16, lphi, flux, steps=1)
    if cfg.rhsc_open:
        cfg.rhsc_open = 0
        o = OracleCy(cfg)
    s = cy.CySolver(cfg)
    du, dbr, dbz = s.lh(uh, br, bz, t)
    edu, edbr, edbz = o.lh(uh.copy(), t)
    assert np.array_equal(du, edu), np.abs(du - edu).max()
    assert np.array_equal(dbr, edbr) and np.array_equal(dbz, edbz)


def test_lh_with_the_manufactured_source_within_tolerance():
    cfg, tend, o, uh, br, bz, t = _state(cy.CY_SIN3D, 16, 12, 2, steps=1)
    s = cy.CySolver(cfg)
    du, dbr, dbz = s.lh(uh, br, bz, 0.37)
    edu, edbr, edbz = o.lh(uh.copy(), 0.37)
    # device sin/cos in S1..S7: 1e-12 of the largest term, relative
    for a, b in ((du, edu), (dbr, edbr), (dbz, edbz)):
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()
    assert not np.array_equal(du, 0 * du)


@pytest.mark.parametrize("problem,lphi", [(cy.CY_ORSZAG_TANG, 1), (cy.CY_ORSZAG_TANG2, 2), (cy.CY_EXPLOSION, 1),
                                          (cy.CY_ROTOR, 1), (cy.CY_JET, 1)])
def test_limit_and_dt_match_oracle(problem, lphi):
    cfg, tend, o, uh, br, bz, t = _state(problem, 20, 16, lphi, steps=1)
    # a pre-limit stage state: one forward-Euler stage of the step
    dt = o.dt(uh)
    du, dbr, dbz = o.lh(uh, t)
    ut, rt, zt = uh + dt * du, br + dt * dbr, bz + dt * dbz
    s = cy.CySolver(cfg)
    assert s.dt(uh) == dt
    ga, gr, gz = ut.copy(), rt.copy(), zt.copy()
    s.limit(ga, gr, gz)
    ea, er, ez = ut.copy(), rt.copy(), zt.copy()
    flags = o.limit(ea, er, ez)
    if problem in (cy.CY_EXPLOSION, cy.CY_ROTOR, cy.CY_ORSZAG_TANG2):
        assert flags.any(), "the case should exercise the limiter"
    assert np.array_equal(_interior(ga), _interior(ea)), np.abs(_interior(ga) - _interior(ea)).max()
    assert np.array_equal(gr, er) and np.array_equal(gz, ez)


@pytest.mark.parametrize("problem,lphi,nr,nz,steps,over", [
    (cy.CY_ORSZAG_TANG, 1, 32, 32, 4, {}),
    (cy.CY_ORSZAG_TANG2, 2, 24, 24, 3, {}),
    (cy.CY_ORSZAG_TANG2, 4, 16, 16, 3, {"flux_type": cy.CY_FLUX_LF}),
    (cy.CY_EXPLOSION, 1, 32, 32, 4, {}),
    (cy.CY_ROTOR, 1, 32, 32, 4, {}),
    (cy.CY_JET, 1, 24, 24, 3, {}),
    (cy.CY_JET, 2, 24, 24, 3, {"bc_d": 4}),
    (cy.CY_EXPLOSION, 1, 24, 24, 3, {"bc_l": 3}),
    (cy.CY_SMOOTH_VORTEX, 1, 24, 24, 1, {"ra": 1.0, "rb": 11.0})])
def test_steps_match_oracle(problem, lphi, nr, nz, steps, over):
    cfg, tend = cy_problem_config(problem, nr, nz, lphi)
    for k, v in over.items():
        setattr(cfg, k, v)
    o = OracleCy(cfg)
    uh, br, bz = o.init_data(problem)
    s = cy.CySolver(cfg)
    s.upload(uh, br, bz)
    s.prepare()
    o.limit(uh, br, bz)
    gu, gr, gz = s.download()
    assert np.array_equal(_interior(gu), _interior(uh)) and np.array_equal(gr, br) and np.array_equal(gz, bz)
    t = 0.0
    for k in range(steps):
        if not t < tend:   # RK3.f90:40: the loop ends once t reaches tend
            break
        t, dt = o.step(uh, br, bz, t, tend)
        gt, gdt = s.step(tend)
        assert gt == t and gdt == dt, (k, gt, t, gdt, dt)
        gu, gr, gz = s.download()
        assert np.array_equal(_interior(gu), _interior(uh)), (k, np.abs(_interior(gu) - _interior(uh)).max())
        assert np.array_equal(gr, br) and np.array_equal(gz, bz), k
    assert np.all(gu[~cy.cy_live_mask()] == 0.0)


def test_manufactured_solution_steps_within_tolerance():
    cfg, tend = cy_problem_config(cy.CY_SIN3D, 16, 16, 4)
    o = OracleCy(cfg)
    uh, br, bz = o.init_data(cy.CY_SIN3D)
    s = cy.CySolver(cfg)
    s.upload(uh, br, bz)
    s.prepare()
    o.limit(uh, br, bz)
    t = 0.0
    for _ in range(3):
        t, dt = o.step(uh, br, bz, t, tend)
        gt, gdt = s.step(tend)
        assert abs(gt - t) <= 1e-14 and abs(gdt - dt) <= 1e-12 * dt
    gu, gr, gz = s.download()
    # device sin/cos in the source: 1e-10 of each variable's scale after three steps
    for n in range(8):
        scale = max(np.abs(uh[n]).max(), 1e-300)
        assert np.abs(gu[n][..., 1:-1, 1:-1] - uh[n][..., 1:-1, 1:-1]).max() <= 1e-10 * scale, n
    assert np.abs(gr - br).max() <= 1e-10 * np.abs(br).max()


def test_advance_replays_equal_single_steps_and_stop_at_tend():
    cfg, _ = cy_problem_config(cy.CY_ROTOR, 24, 24, 1)
    uh, br, bz = cy.cy_init_data(cfg, cy.CY_ROTOR)
    a, b = cy.CySolver(cfg), cy.CySolver(cfg)
    for s in (a, b):
        s.upload(uh, br, bz)
        s.prepare()
    for _ in range(5):
        a.step(1.0)
    t, n = b.advance(1.0, 5)
    assert n == 5 and t == a.t
    ua, ra, za = a.download()
    ub, rb, zb = b.download()
    assert np.array_equal(_interior(ua), _interior(ub)) and np.array_equal(ra, rb) and np.array_equal(za, zb)
    tend = a.t + 1e-4
    t, n = b.advance(tend, 1000)
    assert t == tend and 1 <= n < 1000
    assert b.kernel_launches() > 30 * n


@pytest.mark.parametrize("problem,lphi", [(cy.CY_ORSZAG_TANG, 1), (cy.CY_ORSZAG_TANG2, 2), (cy.CY_ROTOR, 1)])
def test_diagnostics_match_oracle(problem, lphi):
    cfg, tend, o, uh, br, bz, t = _state(problem, 20, 16, lphi, steps=2)
    s = cy.CySolver(cfg)
    s.upload(uh, br, bz)
    umax, totaldiv, pmin = s.diagnostics()
    eu, et, ep = o.diagnostics(uh)
    assert umax == eu and pmin == ep
    assert abs(totaldiv - et) <= 1e-12 * max(et, 1e-300) + 1e-300
    assert totaldiv < 1e-12


def test_orszag_tang_192_reference_configuration_one_step():
    """The reference's own configuration (com.txt:1 Nr = Nz = 192, Lphi = 1,
    HLL; init_data.f90:16 includes init3.txt): one step from the initial
    data."""
    cfg, tend = cy_problem_config(cy.CY_ORSZAG_TANG, 192, 192, 1)
    uh, br, bz = cy.cy_init_data(cfg, cy.CY_ORSZAG_TANG)
    s = cy.CySolver(cfg)
    s.upload(uh, br, bz)
    s.prepare()
    o = OracleCy(cfg)
    o.limit(uh, br, bz)
    t, dt = o.step(uh, br, bz, 0.0, tend)
    gt, gdt = s.step(tend)
    assert gt == t and gdt == dt
    gu, gr, gz = s.download()
    assert np.array_equal(_interior(gu), _interior(uh)) and np.array_equal(gr, br) and np.array_equal(gz, bz)


def test_upload_rejects_a_dead_slot():
    cfg, _ = cy_problem_config(cy.CY_ROTOR, 16, 16, 1)
    uh, br, bz = cy.cy_init_data(cfg, cy.CY_ROTOR)
    uh[0, 7, 0, 5, 5] = 1.0   # mode 8 of rho: the method never fills it
    s = cy.CySolver(cfg)
    import gdf
    with pytest.raises(gdf.GdfError):
        s.upload(uh, br, bz)
