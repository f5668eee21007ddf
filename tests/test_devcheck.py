"""The library's pointwise physics (csrc/gdf_physics.cuh, the code the
sm_100a kernels run) compiled for the host without FMA, compared value for
value with the oracle on random states: Riemann solvers (LF, HLL, HLLC,
HLLD, both directions), fast speeds, eigenmatrix (both directions), and the
2-D vertex solvers."""
import ctypes as C

import numpy as np
import pytest

import gdf
from native_build import build_devcheck
from oracle import Oracle

dp = C.POINTER(C.c_double)


def P(a):
    return np.ascontiguousarray(a, np.float64).ctypes.data_as(dp)


@pytest.fixture(scope="module")
def dev():
    L = C.CDLL(build_devcheck())
    L.dev_vertex_ez.restype = C.c_double
    return L


def rand_state(rng, g):
    rho = 10 ** rng.uniform(-1, 1)
    u = rng.uniform(-3, 3, 3) * (10 if rng.random() < 0.2 else 1)
    B = rng.uniform(-5, 5, 3)
    for k in range(3):
        if rng.random() < 0.3:
            u[k] = 0.0
        if rng.random() < 0.3:
            B[k] = 0.0
    r = rng.random()
    if r < 0.1:      # tangential B below the pick_orthogonal threshold (x normal)
        B[1] = rng.uniform(-1e-4, 1e-4)
        B[2] = 0.0
    elif r < 0.2:    # same for the y normal
        B[0] = rng.uniform(-1e-4, 1e-4)
        B[2] = 0.0
    p = 10 ** rng.uniform(-2, 1)
    E = p / (g - 1) + 0.5 * rho * (u @ u) + 0.5 * (B @ B)
    return (np.array([rho, rho * u[0], rho * u[1], rho * u[2], E, B[0], B[1], B[2]]),
            np.array([rho, *u, E, *B]))


def same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))


VARIANTS = [  # gamma, gamma_flux, hlld_eps, eig_p_typo, eig_identity, kml_w_term
    (5 / 3, 5 / 3, 1e-4, 0, 1, 1),
    (1.4, 5 / 3, 1e-4, 0, 1, 1),
    (1.4, 5 / 3, 1e-12, 1, 0, 0),
    (1.4, 1.4, 1e-6, 0, 1, 1),
]


@pytest.mark.parametrize("flux", [1, 2, 3, 4])
@pytest.mark.parametrize("variant", range(len(VARIANTS)))
def test_pointwise_physics_matches_oracle(dev, flux, variant):
    g, gf, eps, typo, ident, kml = VARIANTS[variant]
    cfg = gdf.reference_config(8, 8)
    cfg.gamma, cfg.gamma_flux, cfg.hlld_eps, cfg.flux_type = g, gf, eps, flux
    cfg.eig_p_typo, cfg.eig_identity, cfg.kml_w_term = typo, ident, kml
    o = Oracle(cfg)
    prm = np.array([g, gf, eps])
    iprm = (C.c_int * 4)(flux, kml, typo, ident)
    rng = np.random.default_rng(100 * flux + variant)
    for _ in range(1500):
        Ua, pa = rand_state(rng, g)
        Ub, _ = rand_state(rng, g)
        for dr in (1, 2):
            f1 = o.riemann(Ua, Ub, dr)
            f2 = np.zeros(8)
            dev.dev_face_flux(P(prm), iprm, P(Ua), P(Ub), dr, P(f2))
            assert same(f1, f2), (flux, dr, Ua, Ub, f1, f2)
            if flux == 2:
                n = [1.0 if dr == 1 else 0.0, 1.0 if dr == 2 else 0.0, 0.0]
                R1, L1 = o.eigenmatrix(pa, n)
                R2 = np.zeros(64)
                L2 = np.zeros(64)
                dev.dev_eigenmatrix(P(prm), iprm, dr, P(pa), P(R2), P(L2))
                assert same(R1, R2.reshape(8, 8).T) and same(L1, L2.reshape(8, 8).T), (dr, pa)
                a1 = o.eigenvalue(Ua, 1 if dr == 1 else 0, 1 if dr == 2 else 0)
                x, y = C.c_double(), C.c_double()
                dev.dev_eigenvalue(P(prm), iprm, P(Ua), dr, C.byref(x), C.byref(y))
                assert same(a1, (x.value, y.value))
        S = [rand_state(rng, g)[0] for _ in range(4)]
        e1 = o.vertex_ez(*S)
        e2 = dev.dev_vertex_ez(P(prm), iprm, *[P(s) for s in S])
        assert same(e1, e2), (flux, S, e1, e2)
