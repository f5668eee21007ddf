"""ctypes mirror of include/gdf.h (the C ABI of the B200 library).

The layout of :class:`GdfConfig` must match ``struct GdfConfig`` field for
field; ``tests/test_abi.py`` checks the size against the C compiler's.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

GDF_OK = 0
GDF_ERR_ARG = 1
GDF_ERR_CUDA = 2
GDF_ERR_NUMERIC = 3
GDF_ERR_TIMEOUT = 4
GDF_ERR_NOMEM = 5
GDF_ERR_STATE = 6

FLUX_LF, FLUX_HLL, FLUX_HLLC, FLUX_HLLD = 1, 2, 3, 4
BC_PERIODIC, BC_OUTFLOW = 1, 2
DETECT_ALL, DETECT_KXRCF = 0, 1
PROB_VORTEX, PROB_ORSZAG_TANG, PROB_ROTOR, PROB_BLAST, PROB_CLOUD_SHOCK = 0, 1, 2, 3, 4

NP = 10  # modal slots per variable (dimPk for k = 2)
NE = 8   # conserved variables


class GdfConfig(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32),
        ("xa", C.c_double), ("xb", C.c_double), ("ya", C.c_double), ("yb", C.c_double),
        ("bc_r", C.c_int32), ("bc_l", C.c_int32), ("bc_u", C.c_int32), ("bc_d", C.c_int32),
        ("gamma", C.c_double), ("gamma_flux", C.c_double),
        ("flux_type", C.c_int32),
        ("cfl", C.c_double), ("tvb_m", C.c_double), ("tvb_slope", C.c_double), ("hlld_eps", C.c_double),
        ("pp_limiter", C.c_int32), ("faceb_limiter", C.c_int32), ("ez_face_fhat", C.c_int32),
        ("eig_p_typo", C.c_int32), ("eig_identity", C.c_int32), ("eig_y_zero_w", C.c_int32),
        ("kml_w_term", C.c_int32), ("dt_floor_stop", C.c_int32), ("umax_all_vars", C.c_int32),
        ("detector", C.c_int32),
        ("kxrcf_ck", C.c_double),
        ("kxrcf_sticky", C.c_int32),
        ("tvb_p1", C.c_int32), ("reserved_i", C.c_int32 * 6),
        ("reserved_d", C.c_double * 4),
    ]

    def copy(self) -> "GdfConfig":
        out = GdfConfig()
        C.memmove(C.byref(out), C.byref(self), C.sizeof(GdfConfig))
        return out

    def as_dict(self) -> dict:
        d = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            if not isinstance(v, (int, float)):
                v = list(v)
            d[name] = v
        return d


def reference_config(nx: int, ny: int) -> GdfConfig:
    """GDF_Balsara_P2_0316 as shipped (com.txt, calculate_dt.f90, the
    commented-out lines of TVB_Limiter_P2.f90), pure-Python twin of
    gdf_config_reference()."""
    c = GdfConfig()
    c.nx, c.ny = nx, ny
    c.xa, c.xb, c.ya, c.yb = 0.0, 1.0, 0.0, 1.0
    c.bc_r = c.bc_l = c.bc_u = c.bc_d = BC_PERIODIC
    c.gamma = 5.0 / 3.0
    c.gamma_flux = 5.0 / 3.0
    c.flux_type = FLUX_HLL
    c.cfl = 0.15
    c.tvb_m = 10.0
    c.tvb_slope = 0.75
    c.hlld_eps = 1e-4
    c.pp_limiter = 0
    c.faceb_limiter = 0
    c.ez_face_fhat = 0
    c.eig_p_typo = 0
    c.eig_identity = 1
    c.eig_y_zero_w = 0
    c.kml_w_term = 1
    c.dt_floor_stop = 1
    c.umax_all_vars = 0
    c.detector = DETECT_ALL
    c.kxrcf_ck = 0.0
    c.kxrcf_sticky = 1
    return c


def problem_config(problem: int, nx: int, ny: int) -> tuple[GdfConfig, float]:
    """Problem presets (pure-Python twin of gdf_problem_config())."""
    c = reference_config(nx, ny)
    pi = 4 * math.atan(1.0)
    if problem == PROB_VORTEX:            # init1.txt
        c.xa, c.xb, c.ya, c.yb = -10.0, 10.0, -10.0, 10.0
        c.tvb_m = 1000000.0
        tend = 0.0
    elif problem == PROB_ORSZAG_TANG:     # init3.txt, M = 50, t = 0.5
        c.xa, c.xb, c.ya, c.yb = 0.0, 2 * pi, 0.0, 2 * pi
        c.tvb_m = 50.0
        tend = 0.5
    elif problem == PROB_ROTOR:           # rotor: HLLD, gamma 1.4, KXRCF + pp, face-B minmod
        c.xa, c.xb, c.ya, c.yb = 0.0, 1.0, 0.0, 1.0
        c.gamma = 1.4
        c.flux_type = FLUX_HLLD
        c.pp_limiter = 1
        c.detector = DETECT_KXRCF
        c.kxrcf_ck = 1.0
        c.tvb_m = 10.0
        c.faceb_limiter = 1                # face-B minmod (raw face B loses positivity near t = 0.013)
        tend = 0.295
    elif problem == PROB_BLAST:           # blast: HLLD, gamma 1.4, pp, outflow
        c.xa, c.xb, c.ya, c.yb = -0.5, 0.5, -0.5, 0.5
        c.bc_r = c.bc_l = c.bc_u = c.bc_d = BC_OUTFLOW
        c.gamma = 1.4
        c.flux_type = FLUX_HLLD
        c.pp_limiter = 1
        c.detector = DETECT_KXRCF
        c.kxrcf_ck = 1.0
        c.tvb_m = 10.0
        c.faceb_limiter = 1                # DF-variant face-B minmod (robustness)
        tend = 0.01
    elif problem == PROB_CLOUD_SHOCK:     # init6.txt (the reference default)
        c.xa, c.xb, c.ya, c.yb = 0.0, 2.0, 0.0, 1.0
        c.bc_r = c.bc_l = c.bc_u = c.bc_d = BC_OUTFLOW
        c.tvb_m = 10.0
        tend = 0.6
    else:
        raise ValueError(f"unknown problem {problem}")
    return c, tend


def uh_shape(nx: int, ny: int) -> tuple:
    """numpy shape (n, d, j, i) of uh(0:Nx+1, 0:Ny+1, 10, 8) in Fortran order."""
    return (NE, NP, ny + 2, nx + 2)


def bx_shape(nx: int, ny: int) -> tuple:
    return (3, ny, nx + 1)


def by_shape(nx: int, ny: int) -> tuple:
    return (3, ny + 1, nx)


def new_state(nx: int, ny: int):
    return (np.zeros(uh_shape(nx, ny)), np.zeros(bx_shape(nx, ny)), np.zeros(by_shape(nx, ny)))


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_double))


def iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_int32))


PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_DIR = os.path.join(PKG_DIR, "lib")
