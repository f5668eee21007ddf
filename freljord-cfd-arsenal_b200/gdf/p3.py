"""The k = 3 variant (MPI_BalsaraP3/main.f90): ctypes mirror of
include/gdf_p3.h and the device-resident solver over it.

Arrays are the reference's per-rank arrays of a single-rank run in Fortran
order, as numpy C-order arrays with the reversed extents:
uh (8, 15, Ny+2, Nx+2), Bx (4, Ny+2, Nx+1), By (4, Ny+1, Nx+2).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from ._abi import (BC_OUTFLOW, BC_PERIODIC, FLUX_HLL, PROB_CLOUD_SHOCK, PROB_ORSZAG_TANG, PROB_ROTOR,
                   PROB_VORTEX, dptr)

NP3 = 15   # modal slots per variable (dimPk for kk = 3)
NB3 = 4    # face modes (kk + 1)
NE = 8

P3_PROBLEMS = (PROB_VORTEX, PROB_ORSZAG_TANG, PROB_ROTOR, PROB_CLOUD_SHOCK)


class GdfP3Config(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32),
        ("xa", C.c_double), ("xb", C.c_double), ("ya", C.c_double), ("yb", C.c_double),
        ("bc_r", C.c_int32), ("bc_l", C.c_int32), ("bc_u", C.c_int32), ("bc_d", C.c_int32),
        ("flux_type", C.c_int32),
        ("gamma", C.c_double), ("cfl", C.c_double), ("tvb_m", C.c_double), ("tvb_beta", C.c_double),
        ("hlld_eps", C.c_double), ("change_tol", C.c_double),
        ("nx_global", C.c_int32), ("ny_global", C.c_int32),
        ("reserved", C.c_int32 * 2),
    ]

    def copy(self) -> "GdfP3Config":
        out = GdfP3Config()
        C.memmove(C.byref(out), C.byref(self), C.sizeof(GdfP3Config))
        return out

    def as_dict(self) -> dict:
        return {name: (getattr(self, name) if name != "reserved" else list(self.reserved))
                for name, _ in self._fields_}


def p3_problem_config(problem: int, nx: int, ny: int) -> tuple[GdfP3Config, float]:
    """Pure-Python twin of gdf_p3_config_problem(): the mesh subroutine of
    the init module (main.f90:126-155 init1, 197-226 init3, 310-339 init4,
    458-489 init6) and the module constants (main.f90:9,19, RK4 CFL :1319)."""
    c = GdfP3Config()
    c.nx, c.ny = nx, ny
    c.flux_type = FLUX_HLL
    c.gamma = 5.0 / 3.0
    c.cfl = 0.75
    c.hlld_eps = 1e-6
    c.change_tol = 1e-13
    c.tvb_beta = 1.0
    pi = 4 * math.atan(1.0)
    if problem == PROB_VORTEX:
        c.xa, c.xb, c.ya, c.yb = -10.0, 10.0, -10.0, 10.0
        bc, tend, c.tvb_m = BC_PERIODIC, 20.0, 100000000.0
    elif problem == PROB_ORSZAG_TANG:
        c.xa, c.xb, c.ya, c.yb = 0.0, 2 * pi, 0.0, 2 * pi
        bc, tend, c.tvb_m = BC_PERIODIC, 3.0, 10.0
    elif problem == PROB_ROTOR:
        c.xa, c.xb, c.ya, c.yb = 0.0, 1.0, 0.0, 1.0
        bc, tend, c.tvb_m = BC_PERIODIC, 0.295, 1.0
        c.tvb_beta = 0.65
    elif problem == PROB_CLOUD_SHOCK:
        c.xa, c.xb, c.ya, c.yb = 0.0, 2.0, 0.0, 1.0
        bc, tend, c.tvb_m = BC_OUTFLOW, 0.6, 1.0
    else:
        raise ValueError(f"problem {problem} has no init module in MPI_BalsaraP3/main.f90")
    c.bc_r = c.bc_l = c.bc_u = c.bc_d = bc
    return c, tend


def p3_uh_shape(nx: int, ny: int) -> tuple:
    return (NE, NP3, ny + 2, nx + 2)


def p3_bx_shape(nx: int, ny: int) -> tuple:
    return (NB3, ny + 2, nx + 1)


def p3_by_shape(nx: int, ny: int) -> tuple:
    return (NB3, ny + 1, nx + 2)


def p3_new_state(nx: int, ny: int):
    return (np.zeros(p3_uh_shape(nx, ny)), np.zeros(p3_bx_shape(nx, ny)), np.zeros(p3_by_shape(nx, ny)))


def p3_live_mask() -> np.ndarray:
    """(8, 15) bool: the slots the method can make non-zero."""
    m = np.zeros((NE, NP3), bool)
    m[:, :10] = True
    m[5, [10, 13]] = True     # cell Bx: a40 (mode 11), a13 (mode 14)
    m[6, [11, 14]] = True     # cell By: b31 (mode 12), b04 (mode 15)
    return m


def _declare(L) -> None:
    if getattr(L, "_gdf_p3_declared", False):
        return
    vp, dp, i32 = C.c_void_p, C.POINTER(C.c_double), C.c_int32
    cp = C.POINTER(GdfP3Config)
    L.gdf_p3_config_problem.argtypes = [i32, i32, i32, cp, dp]
    L.gdf_p3_init_data.argtypes = [cp, i32, dp, dp, dp]
    L.gdf_p3_create.argtypes = [cp, C.POINTER(vp)]
    L.gdf_p3_destroy.argtypes = [vp]
    L.gdf_p3_upload.argtypes = [vp, dp, dp, dp]
    L.gdf_p3_download.argtypes = [vp, dp, dp, dp]
    L.gdf_p3_set_time.argtypes = [vp, C.c_double]
    L.gdf_p3_prepare.argtypes = [vp]
    L.gdf_p3_step.argtypes = [vp, C.c_double, dp, dp]
    L.gdf_p3_advance.argtypes = [vp, C.c_double, i32, dp, C.POINTER(i32)]
    L.gdf_p3_advance_timed.argtypes = [vp, C.c_double, i32, dp, C.POINTER(i32), dp]
    L.gdf_p3_kernel_launches.argtypes = [vp]
    L.gdf_p3_kernel_launches.restype = C.c_int64
    L.gdf_p3_lh.argtypes = [vp, dp, dp, dp, dp, dp, dp]
    L.gdf_p3_limit.argtypes = [vp, dp, dp, dp]
    L.gdf_p3_dt.argtypes = [vp, dp, dp]
    L.gdf_p3_diagnostics.argtypes = [vp, dp, dp]
    pp = C.POINTER(C.c_void_p)
    L.gdf_p3_block_arrays.argtypes = [vp, pp, pp, pp, pp, pp, pp]
    L.gdf_p3_stream.argtypes = [vp]
    L.gdf_p3_stream.restype = C.c_void_p
    L.gdf_p3_step_speeds.argtypes = [vp, dp, dp]
    L.gdf_p3_step_begin.argtypes = [vp, C.c_double, C.c_double, C.c_double, dp, dp]
    L.gdf_p3_stage_lh.argtypes = [vp, i32]
    L.gdf_p3_stage_limit.argtypes = [vp]
    L.gdf_p3_stage_load_t.argtypes = [vp]
    L._gdf_p3_declared = True


def _lib(exact: bool):
    from . import load
    L = load(exact)
    _declare(L)
    return L


def _check(L, rc: int) -> None:
    from . import _check as ck
    ck(L, rc)


def c_p3_problem_config(problem: int, nx: int, ny: int, exact: bool = True):
    """gdf_p3_config_problem through the library."""
    L = _lib(exact)
    c = GdfP3Config()
    tend = C.c_double()
    _check(L, L.gdf_p3_config_problem(problem, nx, ny, C.byref(c), C.byref(tend)))
    return c, tend.value


def p3_init_data(cfg: GdfP3Config, problem: int, exact: bool = True):
    """gdf_p3_init_data: the host projection of the initial data."""
    L = _lib(exact)
    uh, bx, by = p3_new_state(cfg.nx, cfg.ny)
    _check(L, L.gdf_p3_init_data(C.byref(cfg), problem, dptr(uh), dptr(bx), dptr(by)))
    return uh, bx, by


class P3Solver:
    """One device-resident k = 3 problem (a gdf_p3_create handle)."""

    def __init__(self, cfg: GdfP3Config, exact: bool = True):
        self.L = _lib(exact)
        self.cfg = cfg.copy()
        self.nx, self.ny = cfg.nx, cfg.ny
        h = C.c_void_p()
        _check(self.L, self.L.gdf_p3_create(C.byref(self.cfg), C.byref(h)))
        self.h = h
        self.t = 0.0

    def close(self) -> None:
        if getattr(self, "h", None):
            self.L.gdf_p3_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, uh, bx, by) -> None:
        _check(self.L, self.L.gdf_p3_upload(self.h, dptr(uh), dptr(bx), dptr(by)))
        self.t = 0.0

    def download(self):
        uh, bx, by = p3_new_state(self.nx, self.ny)
        _check(self.L, self.L.gdf_p3_download(self.h, dptr(uh), dptr(bx), dptr(by)))
        return uh, bx, by

    def set_time(self, t: float) -> None:
        _check(self.L, self.L.gdf_p3_set_time(self.h, t))
        self.t = t

    def prepare(self) -> None:
        _check(self.L, self.L.gdf_p3_prepare(self.h))

    def step(self, tend: float):
        t = C.c_double(self.t)
        dt = C.c_double()
        _check(self.L, self.L.gdf_p3_step(self.h, tend, C.byref(t), C.byref(dt)))
        self.t = t.value
        return t.value, dt.value

    def advance(self, tend: float, max_steps: int):
        t = C.c_double(self.t)
        n = C.c_int32()
        _check(self.L, self.L.gdf_p3_advance(self.h, tend, max_steps, C.byref(t), C.byref(n)))
        self.t = t.value
        return t.value, n.value

    def advance_timed(self, tend: float, steps: int):
        """(t, steps taken, device ms) of `steps` graph replays."""
        t = C.c_double(self.t)
        n = C.c_int32()
        ms = C.c_double()
        _check(self.L, self.L.gdf_p3_advance_timed(self.h, tend, steps, C.byref(t), C.byref(n), C.byref(ms)))
        self.t = t.value
        return t.value, n.value, ms.value

    def kernel_launches(self) -> int:
        return int(self.L.gdf_p3_kernel_launches(self.h))

    def lh(self, uh, bx, by):
        """Lh of the given state: (du, dbx, dby)."""
        du, dbx, dby = np.zeros_like(uh), np.zeros_like(bx), np.zeros_like(by)
        _check(self.L, self.L.gdf_p3_lh(self.h, dptr(uh), dptr(bx), dptr(by), dptr(du), dptr(dbx), dptr(dby)))
        return du, dbx, dby

    def limit(self, uh, bx, by) -> None:
        """TVB_Limiter then div_free_Balsara, in place."""
        _check(self.L, self.L.gdf_p3_limit(self.h, dptr(uh), dptr(bx), dptr(by)))

    def dt(self, uh) -> float:
        d = C.c_double()
        _check(self.L, self.L.gdf_p3_dt(self.h, dptr(uh), C.byref(d)))
        return d.value

    def diagnostics(self):
        a, b = C.c_double(), C.c_double()
        _check(self.L, self.L.gdf_p3_diagnostics(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    # stage-level control of a block (gdf/p3_dist.py drives it)
    def block_arrays(self) -> dict:
        ptrs = [C.c_void_p() for _ in range(6)]
        _check(self.L, self.L.gdf_p3_block_arrays(self.h, *[C.byref(p) for p in ptrs]))
        return dict(zip(("U", "T", "BX", "BY", "BXT", "BYT"), (p.value for p in ptrs)))

    def stream(self) -> int:
        return int(self.L.gdf_p3_stream(self.h) or 0)

    def step_speeds(self):
        a, b = C.c_double(), C.c_double()
        _check(self.L, self.L.gdf_p3_step_speeds(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def step_begin(self, ax: float, ay: float, tend: float):
        t, dt = C.c_double(), C.c_double()
        _check(self.L, self.L.gdf_p3_step_begin(self.h, ax, ay, tend, C.byref(t), C.byref(dt)))
        self.t = t.value
        return t.value, dt.value

    def stage_lh(self, stage: int) -> None:
        _check(self.L, self.L.gdf_p3_stage_lh(self.h, stage))

    def stage_limit(self) -> None:
        _check(self.L, self.L.gdf_p3_stage_limit(self.h))

    def stage_load_t(self) -> None:
        _check(self.L, self.L.gdf_p3_stage_load_t(self.h))
