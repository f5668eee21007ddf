"""ctypes front of the CPU oracle (oracle/gdf_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
the CPU-baseline leg of bench.py, never by the library. Arrays use the
reference's Fortran layouts through numpy C-order arrays whose shapes are
the reversed Fortran extents (see gdf._abi.uh_shape).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "freljord-cfd-arsenal_b200"))

from gdf._abi import (GdfConfig, dptr, iptr, new_state)  # noqa: E402

LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
COUNT_LIB_PATH = os.path.join(HERE, "_build", "liboracle_count.so")


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None
_count_lib = None


def _declare(L):
    vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int32)
    L.orc_create.restype = vp
    L.orc_create.argtypes = [C.POINTER(GdfConfig)]
    L.orc_destroy.argtypes = [vp]
    L.orc_threads.argtypes = [C.c_int]
    L.orc_threads.restype = C.c_int
    L.orc_init_data.argtypes = [vp, C.c_int, dp, dp, dp, dp]
    L.orc_set_bc.argtypes = [vp, dp]
    L.orc_lh.argtypes = [vp, dp, dp]
    L.orc_lhez.argtypes = [vp, dp, dp, dp]
    L.orc_limit.argtypes = [vp, dp, dp, dp, ip]
    L.orc_div_free.argtypes = [vp, dp, dp, dp]
    L.orc_dt.argtypes = [vp, dp, dp]
    L.orc_prepare.argtypes = [vp, dp, dp, dp, ip]
    L.orc_step.argtypes = [vp, dp, dp, dp, dp, C.c_double, dp, ip]
    L.orc_diagnostics.argtypes = [vp, dp, dp, dp, dp]
    L.orc_reset_trouble.argtypes = [vp]
    L.orc_eigenvalue.argtypes = [vp, dp, C.c_int, C.c_int, dp, dp]
    L.orc_eigenmatrix.argtypes = [vp, dp, dp, dp, dp]
    L.orc_riemann.argtypes = [vp, dp, dp, C.c_int, dp]
    L.orc_vertex_ez.argtypes = [vp, dp, dp, dp, dp]
    L.orc_vertex_ez.restype = C.c_double
    L.orc_pow_hxhy.argtypes = [vp]
    L.orc_pow_hxhy.restype = C.c_double
    return L


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = _declare(C.CDLL(LIB_PATH))
    return _lib


def count_lib():
    """The oracle built on the counting scalar (flopcount.h): same values,
    single-threaded, with a tally of its + - * / and square roots."""
    global _count_lib
    if _count_lib is None:
        if not os.path.exists(COUNT_LIB_PATH):
            build()
        L = _declare(C.CDLL(COUNT_LIB_PATH))
        L.orc_flops.argtypes = [C.POINTER(C.c_uint64)]
        _count_lib = L
    return _count_lib


def set_threads(n: int = 0) -> int:
    return lib().orc_threads(n)


class Oracle:
    """One oracle instance per configuration (holds the sticky KXRCF flags)."""

    def __init__(self, cfg: GdfConfig, counting: bool = False):
        self.cfg = cfg.copy()
        self.nx, self.ny = cfg.nx, cfg.ny
        self.L = count_lib() if counting else lib()
        self.h = self.L.orc_create(C.byref(self.cfg))
        if not self.h:
            raise ValueError("bad oracle configuration")

    def __del__(self):
        h = getattr(self, "h", None)
        if h and getattr(self, "L", None) is not None:
            self.L.orc_destroy(h)
            self.h = None

    def state(self):
        return new_state(self.nx, self.ny)

    def flags(self):
        return np.zeros((self.ny, self.nx), np.int32)

    def init_data(self, problem: int, params=None):
        uh, bx, by = self.state()
        p = None if params is None else dptr(np.ascontiguousarray(params, np.float64))
        self.L.orc_init_data(self.h, problem, p, dptr(uh), dptr(bx), dptr(by))
        return uh, bx, by

    def set_bc(self, uh):
        self.L.orc_set_bc(self.h, dptr(uh))

    def lh(self, uh):
        du = np.zeros_like(uh)
        self.L.orc_lh(self.h, dptr(uh), dptr(du))
        return du

    def lhez(self, uh):
        _, d1, d2 = self.state()
        self.L.orc_lhez(self.h, dptr(uh), dptr(d1), dptr(d2))
        return d1, d2

    def limit(self, uh, bx, by):
        f = self.flags()
        self.L.orc_limit(self.h, dptr(uh), dptr(bx), dptr(by), iptr(f))
        return f

    def div_free(self, uh, bx, by):
        self.L.orc_div_free(self.h, dptr(uh), dptr(bx), dptr(by))

    def dt(self, uh) -> float:
        d = C.c_double()
        self.L.orc_dt(self.h, dptr(uh), C.byref(d))
        return d.value

    def prepare(self, uh, bx, by):
        f = self.flags()
        self.L.orc_prepare(self.h, dptr(uh), dptr(bx), dptr(by), iptr(f))
        return f

    def step(self, uh, bx, by, t: float, tend: float):
        tt = C.c_double(t)
        dt = C.c_double()
        f = self.flags()
        self.L.orc_step(self.h, dptr(uh), dptr(bx), dptr(by), C.byref(tt), tend, C.byref(dt), iptr(f))
        return tt.value, dt.value, f

    def diagnostics(self, uh):
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        self.L.orc_diagnostics(self.h, dptr(uh), C.byref(a), C.byref(b), C.byref(c))
        return a.value, b.value, c.value

    def reset_trouble(self):
        self.L.orc_reset_trouble(self.h)

    # pointwise known-answer entry points
    def eigenvalue(self, U8, n1: int, n2: int):
        a, b = C.c_double(), C.c_double()
        self.L.orc_eigenvalue(self.h, dptr(np.ascontiguousarray(U8, np.float64)), n1, n2, C.byref(a), C.byref(b))
        return a.value, b.value

    def eigenmatrix(self, prim8, n3):
        R = np.zeros(64)
        L = np.zeros(64)
        self.L.orc_eigenmatrix(self.h, dptr(np.ascontiguousarray(prim8, np.float64)),
                              dptr(np.ascontiguousarray(n3, np.float64)), dptr(R), dptr(L))
        return R.reshape(8, 8).T.copy(), L.reshape(8, 8).T.copy()   # row-major R[r, c]

    def riemann(self, ul, ur, direction: int):
        f = np.zeros(8)
        self.L.orc_riemann(self.h, dptr(np.ascontiguousarray(ul, np.float64)),
                          dptr(np.ascontiguousarray(ur, np.float64)), direction, dptr(f))
        return f

    def vertex_ez(self, uru, ulu, urd, uld) -> float:
        a = [dptr(np.ascontiguousarray(v, np.float64)) for v in (uru, ulu, urd, uld)]
        return self.L.orc_vertex_ez(self.h, *a)

    def pow_hxhy(self) -> float:
        return self.L.orc_pow_hxhy(self.h)

    # flop tally of the counting build: (add, mul, div, sqrt, pow) since the
    # last reset
    def flops(self):
        f = (C.c_uint64 * 5)()
        self.L.orc_flops(f)
        return tuple(int(v) for v in f)

    def reset_flops(self):
        self.L.orc_flops_reset()


# ------------------------------------------------ the k = 3 variant (P3) --
from gdf.p3 import GdfP3Config, p3_new_state  # noqa: E402


def _declare_p3(L):
    if getattr(L, "_p3_declared", False):
        return L
    vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int32)
    L.orc_p3_create.restype = vp
    L.orc_p3_create.argtypes = [C.POINTER(GdfP3Config)]
    L.orc_p3_destroy.argtypes = [vp]
    L.orc_p3_init_data.argtypes = [vp, C.c_int, dp, dp, dp]
    L.orc_p3_set_bc.argtypes = [vp, dp, dp, dp]
    L.orc_p3_lh.argtypes = [vp, dp, dp, dp, dp, dp, dp]
    L.orc_p3_limit.argtypes = [vp, dp, dp, dp, ip]
    L.orc_p3_dt.argtypes = [vp, dp, dp]
    L.orc_p3_step.argtypes = [vp, dp, dp, dp, dp, C.c_double, dp]
    L.orc_p3_diagnostics.argtypes = [vp, dp, dp, dp]
    L.orc_p3_basis.argtypes = [vp, dp]
    L._p3_declared = True
    return L


class OracleP3:
    """CPU restatement of MPI_BalsaraP3/main.f90 for one rank."""

    def __init__(self, cfg: GdfP3Config):
        self.cfg = cfg.copy()
        self.nx, self.ny = cfg.nx, cfg.ny
        self.L = _declare_p3(lib())
        self.h = self.L.orc_p3_create(C.byref(self.cfg))
        if not self.h:
            raise ValueError("bad oracle configuration")

    def __del__(self):
        h = getattr(self, "h", None)
        if h and getattr(self, "L", None) is not None:
            self.L.orc_p3_destroy(h)
            self.h = None

    def state(self):
        return p3_new_state(self.nx, self.ny)

    def init_data(self, problem: int):
        uh, bx, by = self.state()
        self.L.orc_p3_init_data(self.h, problem, dptr(uh), dptr(bx), dptr(by))
        return uh, bx, by

    def set_bc(self, uh, bx, by):
        self.L.orc_p3_set_bc(self.h, dptr(uh), dptr(bx), dptr(by))

    def lh(self, uh, bx, by):
        """Lh (set_bc applied to the given arrays in place): du, dbx, dby."""
        du, dbx, dby = np.zeros_like(uh), np.zeros_like(bx), np.zeros_like(by)
        self.L.orc_p3_lh(self.h, dptr(uh), dptr(bx), dptr(by), dptr(du), dptr(dbx), dptr(dby))
        return du, dbx, dby

    def limit(self, uh, bx, by):
        """TVB_Limiter then div_free_Balsara in place; per cell the changed
        variables (bits 0-7) and those given the P3 reconstruction (8-15)."""
        f = np.zeros((self.ny, self.nx), np.int32)
        self.L.orc_p3_limit(self.h, dptr(uh), dptr(bx), dptr(by), iptr(f))
        return f

    def dt(self, uh) -> float:
        d = C.c_double()
        self.L.orc_p3_dt(self.h, dptr(uh), C.byref(d))
        return d.value

    def step(self, uh, bx, by, t: float, tend: float):
        tt = C.c_double(t)
        dt = C.c_double()
        self.L.orc_p3_step(self.h, dptr(uh), dptr(bx), dptr(by), C.byref(tt), tend, C.byref(dt))
        return tt.value, dt.value

    def diagnostics(self, uh):
        a, b = C.c_double(), C.c_double()
        self.L.orc_p3_diagnostics(self.h, dptr(uh), C.byref(a), C.byref(b))
        return a.value, b.value

    def basis(self) -> dict:
        out = np.zeros(3 * 25 * 15 + 4 * 5 * 15 + 5 * 15)
        self.L.orc_p3_basis(self.h, dptr(out))
        o = 0
        res = {}
        for k in ("phiG", "phixG", "phiyG"):
            res[k] = out[o:o + 375].reshape(5, 5, 15); o += 375
        for k in ("phiGR", "phiGL", "phiGU", "phiGD"):
            res[k] = out[o:o + 75].reshape(5, 15); o += 75
        for k in ("phiRU", "phiLU", "phiRD", "phiLD", "mm"):
            res[k] = out[o:o + 15].copy(); o += 15
        return res


# ----------------------------------------------- the cylindrical variant --
from gdf.cy import GdfCyConfig, cy_new_state  # noqa: E402


def _declare_cy(L):
    if getattr(L, "_cy_declared", False):
        return L
    vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int32)
    L.orc_cy_create.restype = vp
    L.orc_cy_create.argtypes = [C.POINTER(GdfCyConfig)]
    L.orc_cy_destroy.argtypes = [vp]
    L.orc_cy_init_data.argtypes = [vp, C.c_int, dp, dp, dp]
    L.orc_cy_set_bc.argtypes = [vp, dp]
    L.orc_cy_lh.argtypes = [vp, dp, C.c_double, dp, dp, dp]
    L.orc_cy_limit.argtypes = [vp, dp, dp, dp, ip]
    L.orc_cy_dt.argtypes = [vp, dp, dp]
    L.orc_cy_step.argtypes = [vp, dp, dp, dp, dp, C.c_double, dp]
    L.orc_cy_diagnostics.argtypes = [vp, dp, dp, dp, dp]
    L.orc_cy_l2_error.argtypes = [vp, C.c_int, dp, C.c_double, dp]
    L._cy_declared = True
    return L


class OracleCy:
    """CPU restatement of MHD_GDF_cy3D_0421/ (Lh, LhEz, TVB_Limiter_P2,
    div_free_Balsara, set_bc, calculate_dt, RK3, the diagnostics)."""

    def __init__(self, cfg: GdfCyConfig):
        self.cfg = cfg.copy()
        self.nr, self.nz, self.lphi = cfg.nr, cfg.nz, cfg.lphi
        self.L = _declare_cy(lib())
        self.h = self.L.orc_cy_create(C.byref(self.cfg))
        if not self.h:
            raise ValueError("bad oracle configuration")

    def __del__(self):
        h = getattr(self, "h", None)
        if h and getattr(self, "L", None) is not None:
            self.L.orc_cy_destroy(h)
            self.h = None

    def state(self):
        return cy_new_state(self.nr, self.nz, self.lphi)

    def init_data(self, problem: int):
        uh, br, bz = self.state()
        self.L.orc_cy_init_data(self.h, problem, dptr(uh), dptr(br), dptr(bz))
        return uh, br, bz

    def set_bc(self, uh):
        self.L.orc_cy_set_bc(self.h, dptr(uh))

    def lh(self, uh, t_rk: float = 0.0):
        """Lh then LhEz (set_bc applied to uh in place): du, dbr, dbz."""
        _, br, bz = self.state()
        du, dbr, dbz = np.zeros_like(uh), np.zeros_like(br), np.zeros_like(bz)
        self.L.orc_cy_lh(self.h, dptr(uh), t_rk, dptr(du), dptr(dbr), dptr(dbz))
        return du, dbr, dbz

    def limit(self, uh, br, bz):
        """TVB_Limiter_P2 then div_free_Balsara in place; per cell plane
        (NPH, Nz, Nr) the changed variables (bits 0-7)."""
        f = np.zeros((2 * self.lphi, self.nz, self.nr), np.int32)
        self.L.orc_cy_limit(self.h, dptr(uh), dptr(br), dptr(bz), iptr(f))
        return f

    def dt(self, uh) -> float:
        d = C.c_double()
        self.L.orc_cy_dt(self.h, dptr(uh), C.byref(d))
        return d.value

    def step(self, uh, br, bz, t: float, tend: float):
        tt = C.c_double(t)
        dt = C.c_double()
        self.L.orc_cy_step(self.h, dptr(uh), dptr(br), dptr(bz), C.byref(tt), tend, C.byref(dt))
        return tt.value, dt.value

    def diagnostics(self, uh):
        a, b, p = C.c_double(), C.c_double(), C.c_double()
        self.L.orc_cy_diagnostics(self.h, dptr(uh), C.byref(a), C.byref(b), C.byref(p))
        return a.value, b.value, p.value

    def l2_error(self, problem: int, uh, t: float) -> np.ndarray:
        """calculate_L2_error.f90 against the problem's data translated by
        (t, t): the exact solution of the manufactured problem init1.txt."""
        out = np.zeros(8)
        self.L.orc_cy_l2_error(self.h, problem, dptr(uh), t, dptr(out))
        return out
