"""Committed golden fixtures (tests/golden/*.npz, written by
tests/golden/make_golden.py from the CPU oracle): the oracle must still
reproduce them value for value (CPU), and the sm_100a library must too
(GPU), so the GPU parity holds without building the oracle."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import gdf  # noqa: E402
from make_golden import CASES, case_config  # noqa: E402

NAMES = sorted(CASES)


def load(name):
    return dict(np.load(os.path.join(HERE, "golden", name + ".npz")))


def same(a, b):
    return bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))


@pytest.mark.parametrize("name", NAMES)
def test_fixture_is_well_formed(name):
    g = load(name)
    cfg, prob, steps = case_config(name)
    assert g["uh"].shape == gdf.uh_shape(cfg.nx, cfg.ny)
    assert g["flags"].shape == (steps + 1, cfg.ny, cfg.nx)
    assert np.all(np.diff(g["t"]) > 0) and np.all(g["dt"] > 0)
    uh0, bx0, by0 = gdf.init_data(cfg, prob)
    # the library's host-side initial data equals the oracle's
    assert same(uh0, g["uh0"]) and same(bx0, g["bx0"]) and same(by0, g["by0"])


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_fixture(name):
    from make_golden import run_oracle
    r = run_oracle(name)
    g = load(name)
    for k in ("uh", "bx", "by", "flags", "t", "dt"):
        assert same(r[k], g[k]), k


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_library_reproduces_fixture(name):
    g = load(name)
    cfg, prob, steps = case_config(name)
    s = gdf.Solver(cfg)
    s.upload(g["uh0"], g["bx0"], g["by0"])
    f = s.prepare()
    assert np.array_equal(f, g["flags"][0])
    for k in range(steps):
        t, dt, f = s.step(1e9)
        assert t == g["t"][k] and dt == g["dt"][k]
        assert np.array_equal(f, g["flags"][k + 1])
    uh, bx, by = s.download()
    assert same(uh, g["uh"]) and same(bx, g["bx"]) and same(by, g["by"])
