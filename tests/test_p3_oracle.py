"""The k = 3 variant (MPI_BalsaraP3/main.f90) on the CPU: the oracle's own
pins and the library's host-only P3 entry points.

The reference ships no tests or golden vectors for this variant either; the
oracle's restatement is pinned by what the method itself guarantees:
- get_basis: the tables are the scaled Legendre products and their traces
  (checked against numpy polynomials), orthogonal under the 5x5 Gauss rule
  with the mass matrix mm;
- the smooth vortex (module init1, calculate_L2_Error's exact solution)
  converges at fourth order;
- div_free_Balsara keeps totaldiv at round-off on discontinuous problems;
- the limiter and the Riemann fluxes conserve the cell means of rho, rho u
  and E on a periodic grid.
"""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import gdf
from gdf import p3
from gdf.p3 import GdfP3Config, p3_problem_config
from oracle import OracleP3

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "gdf_p3.h")
P3_PROBLEMS = [gdf.PROB_VORTEX, gdf.PROB_ORSZAG_TANG, gdf.PROB_ROTOR, gdf.PROB_CLOUD_SHOCK]

LAM = np.array([-0.9061798459386639927976269, -0.5384693101056830910363144, 0.0,
                0.5384693101056830910363144, 0.9061798459386639927976269])
WTS = np.array([0.2369268850561890875142640, 0.4786286704993664680412915, 0.5688888888888888888888889,
                0.4786286704993664680412915, 0.2369268850561890875142640])


def _legendre(k):
    """Monic-scaled Legendre polynomials of the basis: 1, x, x^2-1/3,
    x^3-3x/5, x^4-6x^2/7+3/35."""
    c = [[1.0], [0.0, 1.0], [-1 / 3, 0.0, 1.0], [0.0, -3 / 5, 0.0, 1.0], [3 / 35, 0.0, -6 / 7, 0.0, 1.0]][k]
    return np.polynomial.Polynomial(c)


# (degree in x, degree in y) of modes 1..15 (get_basis, main.f90:912-1087)
DEG = [(0, 0), (1, 0), (0, 1), (2, 0), (1, 1), (0, 2), (3, 0), (2, 1), (1, 2), (0, 3), (4, 0), (3, 1), (2, 2),
       (1, 3), (0, 4)]


def test_basis_tables_are_scaled_legendre_products():
    cfg, _ = p3_problem_config(gdf.PROB_ORSZAG_TANG, 16, 12)
    o = OracleP3(cfg)
    B = o.basis()
    hx1 = 0.5 * (cfg.xb - cfg.xa) / cfg.nx
    hy1 = 0.5 * (cfg.yb - cfg.ya) / cfg.ny
    for d, (px, py) in enumerate(DEG):
        Px, Py = _legendre(px), _legendre(py)
        dPx, dPy = Px.deriv(), Py.deriv()
        G = np.outer(Px(LAM), Py(LAM))
        np.testing.assert_allclose(B["phiG"][:, :, d], G, rtol=0, atol=1e-15)
        np.testing.assert_allclose(B["phixG"][:, :, d], np.outer(dPx(LAM), Py(LAM)) / hx1, rtol=1e-14, atol=1e-13)
        np.testing.assert_allclose(B["phiyG"][:, :, d], np.outer(Px(LAM), dPy(LAM)) / hy1, rtol=1e-14, atol=1e-13)
        np.testing.assert_allclose(B["phiGR"][:, d], Px(1.0) * Py(LAM), atol=1e-15)
        np.testing.assert_allclose(B["phiGL"][:, d], Px(-1.0) * Py(LAM), atol=1e-15)
        np.testing.assert_allclose(B["phiGU"][:, d], Px(LAM) * Py(1.0), atol=1e-15)
        np.testing.assert_allclose(B["phiGD"][:, d], Px(LAM) * Py(-1.0), atol=1e-15)
        for key, (sx, sy) in (("phiRU", (1, 1)), ("phiLU", (-1, 1)), ("phiRD", (1, -1)), ("phiLD", (-1, -1))):
            assert abs(B[key][d] - Px(sx) * Py(sy)) < 1e-15, (key, d)
    # orthogonality under the 5x5 rule (exact for degree <= 9): mm is the diagonal
    W = 0.25 * np.outer(WTS, WTS)
    M = np.einsum("ab,abd,abe->de", W, B["phiG"], B["phiG"])
    np.testing.assert_allclose(M, np.diag(B["mm"]), rtol=0, atol=1e-15)


def test_vortex_converges_at_fourth_order():
    """init1's vortex moves by (t, t); the projection of the moved vortex
    (the oracle's init_data on the shifted domain) is the exact answer."""
    T = 1.0
    errs = []
    for n in (16, 32):
        cfg, _ = p3_problem_config(gdf.PROB_VORTEX, n, n)
        o = OracleP3(cfg)
        uh, bx, by = o.init_data(gdf.PROB_VORTEX)
        o.limit(uh, bx, by)
        t = 0.0
        while t < T:
            t, _ = o.step(uh, bx, by, t, T)
        ce = cfg.copy()
        ce.xa, ce.xb, ce.ya, ce.yb = ce.xa - T, ce.xb - T, ce.ya - T, ce.yb - T
        ue, _, _ = OracleP3(ce).init_data(gdf.PROB_VORTEX)
        e = np.abs(uh[[1, 2, 4, 5, 6], 0, 1:-1, 1:-1] - ue[[1, 2, 4, 5, 6], 0, 1:-1, 1:-1]).mean(axis=(1, 2))
        errs.append(e)
    order = np.log2(errs[0] / errs[1])
    print("\nvortex L1 orders (rho u, rho v, E, Bx, By):", np.round(order, 2))
    assert np.all(order > 3.6), order


@pytest.mark.parametrize("problem", [gdf.PROB_ORSZAG_TANG, gdf.PROB_ROTOR, gdf.PROB_CLOUD_SHOCK])
def test_div_free_and_conservation(problem):
    cfg, tend = p3_problem_config(problem, 20, 16)
    o = OracleP3(cfg)
    uh, bx, by = o.init_data(problem)
    o.limit(uh, bx, by)
    means0 = uh[[0, 1, 2, 4], 0, 1:-1, 1:-1].sum(axis=(1, 2))
    t = 0.0
    for _ in range(3):
        t, dt = o.step(uh, bx, by, t, tend)
        assert dt > 0 and np.isfinite(uh).all()
        umax, totaldiv = o.diagnostics(uh)
        assert totaldiv < 1e-12, totaldiv
    if cfg.bc_r == gdf.BC_PERIODIC:
        means = uh[[0, 1, 2, 4], 0, 1:-1, 1:-1].sum(axis=(1, 2))
        scale = np.abs(uh[[0, 1, 2, 4], 0, 1:-1, 1:-1]).sum(axis=(1, 2))
        assert np.all(np.abs(means - means0) <= 1e-12 * scale), (means - means0) / scale


def test_dead_slots_stay_zero_and_ghosts_follow_set_bc():
    cfg, tend = p3_problem_config(gdf.PROB_CLOUD_SHOCK, 16, 12)
    o = OracleP3(cfg)
    uh, bx, by = o.init_data(gdf.PROB_CLOUD_SHOCK)
    o.limit(uh, bx, by)
    t = 0.0
    for _ in range(2):
        t, _ = o.step(uh, bx, by, t, tend)
    live = p3.p3_live_mask()
    assert np.all(uh[~live] == 0.0)
    u = uh.copy()
    o.set_bc(u, bx.copy(), by.copy())
    # outflow: ghost column 0 copies column 1, ghost row 0 copies row 1 (corners from the row pass)
    assert np.array_equal(u[:, :, :, 0], u[:, :, :, 1])
    assert np.array_equal(u[:, :, 0, :], u[:, :, 1, :])
    assert np.array_equal(u[:, :, -1, :], u[:, :, -2, :])


# ---------------------------------------------------------------- C ABI ---

def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gdf_p3_[a-z_0-9]+)\s*\(", src)))


@pytest.mark.parametrize("exact", [False, True])
def test_every_p3_symbol_is_exported(exact):
    lib = gdf.LIB_EXACT if exact else gdf.LIB_FMA
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (gdf_\w+)", out))
    syms = declared_symbols()
    assert len(syms) >= 15
    assert not [s for s in syms if s not in exported]


def test_p3_config_struct_layout_matches_c(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text('#include <stddef.h>\n#include "gdf_p3.h"\n'
                   "size_t cfg_size(void){return sizeof(GdfP3Config);}\n"
                   "size_t off_gamma(void){return offsetof(GdfP3Config, gamma);}\n"
                   "size_t off_tol(void){return offsetof(GdfP3Config, change_tol);}\n")
    so = tmp_path / "sz.so"
    subprocess.run(["gcc", "-shared", "-fPIC", "-I", os.path.join(REPO, "include"), "-o", str(so), str(src)],
                   check=True)
    L = C.CDLL(str(so))
    for f in (L.cfg_size, L.off_gamma, L.off_tol):
        f.restype = C.c_size_t
    assert L.cfg_size() == C.sizeof(GdfP3Config)
    assert L.off_gamma() == GdfP3Config.gamma.offset
    assert L.off_tol() == GdfP3Config.change_tol.offset


@pytest.mark.parametrize("problem", P3_PROBLEMS)
def test_p3_presets_and_init_match_the_oracle_bitwise(problem):
    c_py, t_py = p3_problem_config(problem, 24, 20)
    c_c, t_c = p3.c_p3_problem_config(problem, 24, 20)
    assert bytes(c_py) == bytes(c_c) and t_py == t_c
    uh, bx, by = p3.p3_init_data(c_c, problem)
    ou, ob, oy = OracleP3(c_py).init_data(problem)
    assert np.array_equal(uh, ou) and np.array_equal(bx, ob) and np.array_equal(by, oy)


def test_p3_host_entry_points_reject_bad_arguments():
    L = p3._lib(True)
    c = GdfP3Config()
    assert L.gdf_p3_config_problem(gdf.PROB_BLAST, 16, 16, C.byref(c), None) == gdf._abi.GDF_ERR_ARG
    assert L.gdf_p3_config_problem(gdf.PROB_ROTOR, 1, 16, C.byref(c), None) == gdf._abi.GDF_ERR_ARG
    cfg, _ = p3_problem_config(gdf.PROB_ROTOR, 8, 8)
    uh, bx, by = p3.p3_new_state(8, 8)
    assert L.gdf_p3_init_data(C.byref(cfg), gdf.PROB_BLAST, gdf.dptr(uh), gdf.dptr(bx), gdf.dptr(by)) == \
        gdf._abi.GDF_ERR_ARG
