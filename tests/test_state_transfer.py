"""gdf_upload_state / gdf_download_state: the step state in its smallest
form (modes 1-6 of variables 1-5 and 8 over the interior cells, plus the
face fields). The device rebuilds the rest of uh: the cell Bx/By modes by
the div-free reconstruction (div_free_Balsara.f90:13-79) and the ghosts by
set_bc (set_bc.f90:5-27, ghost B modes cleared as div_free_Balsara.f90:11
leaves them). Checked through the C ABI, value for value:
  * the packed layout is the interior of uh's planes;
  * after a step, download_state + upload_state gives back the whole uh,
    ghosts included, bit for bit;
  * steps taken with a host round trip of the compact state every step
    equal the steps of a resident handle, and equal the oracle's.
The three problems cover the limiter forms: Orszag-Tang (HLL, div-free
fused into the limiter), the rotor (HLLD, KXRCF second pass, face-B
minmod, positivity limiter) and the blast with the learned gate."""
import numpy as np
import pytest

import gdf
from oracle import Oracle

pytestmark = pytest.mark.gpu

STATE_VARS = [0, 1, 2, 3, 4, 7]


def _setup(problem, nx, ny, learned=False):
    cfg, _ = gdf.problem_config(problem, nx, ny)
    net = None
    if learned:
        from gdf.indicator import load_net
        net, lo, hi = load_net()
        cfg.detector = gdf.DETECT_LEARNED
    uh, bx, by = gdf.init_data(cfg, problem)
    solvers = []
    for _ in range(2):
        s = gdf.Solver(cfg)
        if learned:
            s.set_indicator(net, lo, hi)
        s.upload(uh, bx, by)
        s.prepare()
        solvers.append(s)
    return cfg, uh, bx, by, solvers


CASES = [(gdf.PROB_ORSZAG_TANG, 24, 20, False), (gdf.PROB_ROTOR, 40, 36, False), (gdf.PROB_BLAST, 36, 28, True)]


@pytest.mark.parametrize("problem,nx,ny,learned", CASES)
def test_round_trip_every_step_equals_resident(problem, nx, ny, learned):
    cfg, _, _, _, (a, b) = _setup(problem, nx, ny, learned)
    for k in range(4):
        cells, bx, by = b.download_state()
        b.upload_state(cells, bx, by)
        ta, dta, fa = a.step(1e9)
        tb, dtb, fb = b.step(1e9)
        assert dta == dtb and ta == tb, f"step {k}"
        assert np.array_equal(fa, fb), f"troubled-cell words, step {k}"
        ua, bxa, bya = a.download()
        ub, bxb, byb = b.download()
        assert np.array_equal(ua, ub) and np.array_equal(bxa, bxb) and np.array_equal(bya, byb), f"step {k}"


@pytest.mark.parametrize("problem,nx,ny,learned", CASES)
def test_compact_state_rebuilds_the_whole_array(problem, nx, ny, learned):
    cfg, _, _, _, (a, _) = _setup(problem, nx, ny, learned)
    a.step(1e9)
    uh, bx, by = a.download()
    cells, cbx, cby = a.download_state()
    # the packed layout: the interior of the six variables' first six modes
    assert cells.shape == (6, 6, ny, nx)
    assert np.array_equal(cells, uh[STATE_VARS, :6, 1:-1, 1:-1])
    assert np.array_equal(cbx, bx) and np.array_equal(cby, by)
    # wipe the resident state with another one, then rebuild from the packed form
    a.upload(*gdf.init_data(cfg, problem))
    a.upload_state(cells, cbx, cby)
    uh2, bx2, by2 = a.download()
    assert np.array_equal(uh2, uh), "uh rebuilt from the compact state differs"
    assert np.array_equal(bx2, bx) and np.array_equal(by2, by)


def test_round_trip_steps_equal_the_oracle():
    problem = gdf.PROB_ROTOR
    cfg, _ = gdf.problem_config(problem, 32, 28)
    uh, bx, by = gdf.init_data(cfg, problem)
    s = gdf.Solver(cfg)
    s.upload(uh, bx, by)
    s.prepare()
    o = Oracle(cfg)
    o.prepare(uh, bx, by)
    t = 0.0
    for _ in range(3):
        cells, cbx, cby = s.download_state()
        s.upload_state(cells, cbx, cby)
        s.step(1e9)
        t, _, _ = o.step(uh, bx, by, t, 1e9)
    ug, bxg, byg = s.download()
    assert np.array_equal(ug, uh) and np.array_equal(bxg, bx) and np.array_equal(byg, by)


def test_state_calls_reject_null_and_unuploaded():
    cfg, _ = gdf.problem_config(gdf.PROB_ORSZAG_TANG, 16, 16)
    s = gdf.Solver(cfg)
    cells = np.zeros(s.state_shape())
    _, bx, by = gdf._abi.new_state(16, 16)
    with pytest.raises(gdf.GdfError) as e:
        s.download_state(cells, bx, by)
    assert e.value.code == gdf._abi.GDF_ERR_STATE
    rc = s.L.gdf_upload_state(s.h, None, None, None)
    assert rc == gdf._abi.GDF_ERR_ARG
