"""The cylindrical variant (MHD_GDF_cy3D_0421/) on the CPU: the oracle's own
pins and the library's host-only entry points.

The reference ships no tests or golden vectors for this variant. The
oracle's restatement is pinned by what the reference itself provides and
what the method guarantees:
- init1.txt with Source.f90 is a manufactured solution (the initial data
  translated by (t, t), calculate_L2_error.f90); with 2*Lphi = 8 phi planes
  (the phi fluxes carry products of cos(phi) modes, mode 2, which 4 planes
  alias to their Nyquist mode) every variable converges at third order;
- div_free_Balsara keeps the discrete divergence, d(Bphi)/dphi included,
  at round-off once the planes resolve the field's phi modes (Lphi >= 2 for
  init1, init2, init4); with Lphi = 1 the phi derivative of cos(phi) is
  zero on the planes 0 and pi and init1's divergence is O(1), as in the
  reference;
- set_bc's mirror, periodic, scaled-periodic and inlet ghosts.
"""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import gdf
from gdf import cy
from gdf.cy import GdfCyConfig, cy_problem_config
from oracle import OracleCy

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "gdf_cy.h")


def _run(o, uh, br, bz, tend):
    t, k = 0.0, 0
    while t < tend:
        t, _ = o.step(uh, br, bz, t, tend)
        k += 1
    return t, k


def test_manufactured_solution_converges_at_third_order():
    T = 0.05
    errs = []
    for n in (8, 16, 32):
        cfg, _ = cy_problem_config(cy.CY_SIN3D, n, n, 4)
        o = OracleCy(cfg)
        uh, br, bz = o.init_data(cy.CY_SIN3D)
        o.limit(uh, br, bz)
        t, _ = _run(o, uh, br, bz, T)
        assert t == T
        errs.append(o.l2_error(cy.CY_SIN3D, uh, t))
    errs = np.array(errs)
    order = np.log2(errs[1] / errs[2])
    # rho, rho u, rho v, E, B_r, B_z, B_phi (rho w stays at the 1e-6 level of its exact zero)
    for n in (0, 1, 2, 4, 5, 6, 7):
        assert order[n] > 2.6, (n, order)
    assert errs[2][[0, 1, 2, 4]].max() < 1e-4


@pytest.mark.parametrize("problem", [cy.CY_SIN3D, cy.CY_DIV_TEST, cy.CY_ORSZAG_TANG2])
def test_reconstruction_is_divergence_free_when_the_planes_resolve_phi(problem):
    for lphi in (2, 4):
        cfg, _ = cy_problem_config(problem, 16, 12, lphi)
        o = OracleCy(cfg)
        uh, br, bz = o.init_data(problem)
        o.limit(uh, br, bz)
        assert o.diagnostics(uh)[1] < 1e-14
    cfg, _ = cy_problem_config(cy.CY_SIN3D, 16, 12, 1)
    o = OracleCy(cfg)
    uh, br, bz = o.init_data(cy.CY_SIN3D)
    o.limit(uh, br, bz)
    assert o.diagnostics(uh)[1] > 1e-3   # cos(phi) on the planes 0, pi: d/dphi is 0 there


@pytest.mark.parametrize("problem", [cy.CY_ORSZAG_TANG, cy.CY_EXPLOSION, cy.CY_ROTOR, cy.CY_JET])
def test_axisymmetric_runs_stay_divergence_free_and_live_slots_only(problem):
    cfg, tend = cy_problem_config(problem, 20, 16, 1)
    o = OracleCy(cfg)
    uh, br, bz = o.init_data(problem)
    o.limit(uh, br, bz)
    t = 0.0
    for _ in range(3):
        t, _ = o.step(uh, br, bz, t, tend)
    assert np.isfinite(uh).all()
    assert o.diagnostics(uh)[1] < 1e-13
    live = cy.cy_live_mask()
    assert np.all(uh[~live] == 0.0)


def test_set_bc_ghosts():
    # mirror extension (bc 2) flips modes 2 and 5 and copies rows
    cfg, _ = cy_problem_config(cy.CY_ROTOR, 8, 6, 1)
    o = OracleCy(cfg)
    rng = np.random.default_rng(3)
    uh, _, _ = o.state()
    live = cy.cy_live_mask()
    uh[live] = rng.normal(size=uh[live].shape)
    o.set_bc(uh)
    sgn = np.ones(10)
    sgn[[1, 4]] = -1
    assert np.array_equal(uh[:, :6, :, 1:-1, -1], uh[:, :6, :, 1:-1, -2] * sgn[None, :6, None, None])
    assert np.array_equal(uh[:, :, :, 0, :], uh[:, :, :, 1, :])
    # periodic with r*B rescaled (bc 4)
    cfg, _ = cy_problem_config(cy.CY_ORSZAG_TANG2, 8, 6, 2)
    o = OracleCy(cfg)
    uh, _, _ = o.state()
    uh[live] = rng.normal(size=uh[live].shape)
    o.set_bc(uh)
    assert np.array_equal(uh[:5, :, :, 1:-1, -1], uh[:5, :, :, 1:-1, 1])
    assert np.array_equal(uh[5:7, :, :, 1:-1, -1], uh[5:7, :, :, 1:-1, 1] * cfg.rb / cfg.ra)
    # the jet inlet (bc_d 4) keeps only the cell means of the inlet cells
    cfg, _ = cy_problem_config(cy.CY_JET, 8, 6, 1)
    cfg.bc_d = 4
    o = OracleCy(cfg)
    uh, _, _ = o.state()
    uh[live] = rng.normal(size=uh[live].shape)
    o.set_bc(uh)
    inlet = [i for i in range(1, 9) if cfg.ra + i * (cfg.rb - cfg.ra) / 8 <= cfg.jet_r]
    outside = [i for i in range(1, 9) if i not in inlet]
    assert inlet and outside and np.all(uh[:, 1:, :, 0, inlet] == 0.0)
    assert np.array_equal(uh[:, :, :, 0, outside], uh[:, :, :, 1, outside])


# ---------------------------------------------------------------- C ABI ---

def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gdf_cy_[a-z_0-9]+)\s*\(", src)))


@pytest.mark.parametrize("exact", [False, True])
def test_every_cy_symbol_is_exported(exact):
    lib = gdf.LIB_EXACT if exact else gdf.LIB_FMA
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (gdf_\w+)", out))
    syms = declared_symbols()
    assert len(syms) >= 16
    assert not [s for s in syms if s not in exported]


def test_cy_config_struct_layout_matches_c(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text('#include <stddef.h>\n#include "gdf_cy.h"\n'
                   "size_t cfg_size(void){return sizeof(GdfCyConfig);}\n"
                   "size_t off_ra(void){return offsetof(GdfCyConfig, ra);}\n"
                   "size_t off_jet(void){return offsetof(GdfCyConfig, jet_r);}\n")
    so = tmp_path / "sz.so"
    subprocess.run(["gcc", "-shared", "-fPIC", "-I", os.path.join(REPO, "include"), "-o", str(so), str(src)],
                   check=True)
    L = C.CDLL(str(so))
    for f in (L.cfg_size, L.off_ra, L.off_jet):
        f.restype = C.c_size_t
    assert L.cfg_size() == C.sizeof(GdfCyConfig)
    assert L.off_ra() == GdfCyConfig.ra.offset
    assert L.off_jet() == GdfCyConfig.jet_r.offset


@pytest.mark.parametrize("problem", cy.CY_PROBLEMS)
def test_cy_presets_and_init_match_the_oracle_bitwise(problem):
    for lphi in (1, 2):
        c_py, t_py = cy_problem_config(problem, 12, 10, lphi)
        c_c, t_c = cy.c_cy_problem_config(problem, 12, 10, lphi)
        assert bytes(c_py) == bytes(c_c) and t_py == t_c
        uh, br, bz = cy.cy_init_data(c_c, problem)
        ou, ob, oz = OracleCy(c_py).init_data(problem)
        assert np.array_equal(uh, ou) and np.array_equal(br, ob) and np.array_equal(bz, oz)
        assert np.all(uh[~cy.cy_live_mask()] == 0.0)


def test_cy_host_entry_points_reject_bad_arguments():
    L = cy._lib(True)
    c = GdfCyConfig()
    assert L.gdf_cy_config_problem(8, 16, 16, 1, C.byref(c), None) == gdf._abi.GDF_ERR_ARG
    assert L.gdf_cy_config_problem(cy.CY_ROTOR, 16, 16, 3, C.byref(c), None) == gdf._abi.GDF_ERR_ARG
    assert L.gdf_cy_config_problem(cy.CY_ROTOR, 1, 16, 1, C.byref(c), None) == gdf._abi.GDF_ERR_ARG
    cfg, _ = cy_problem_config(cy.CY_ROTOR, 8, 8, 1)
    uh, br, bz = cy.cy_new_state(8, 8, 1)
    assert L.gdf_cy_init_data(C.byref(cfg), 9, gdf.dptr(uh), gdf.dptr(br), gdf.dptr(bz)) == gdf._abi.GDF_ERR_ARG
    with pytest.raises(ValueError):
        cy_problem_config(8, 8, 8)
