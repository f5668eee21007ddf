"""The cylindrical variant (MHD_GDF_cy3D_0421/): ctypes mirror of
include/gdf_cy.h and the device-resident solver over it.

Arrays are the reference's COMMON arrays (com.txt:36-68) in Fortran order,
as numpy C-order arrays with the reversed extents (NPH = 2*Lphi planes):
uh (8, 10, NPH, Nz+2, Nr+2), Br (3, NPH, Nz, Nr+1), Bz (3, NPH, Nz+1, Nr).
uh[5], uh[6] hold r*B_r and r*B_z; Br and Bz hold r*B on the faces.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from ._abi import dptr

NPC = 10   # modal slots per variable (dimPk for k = 2)
NQC = 6    # P2 test functions (dimPk1)
NE = 8

CY_SMOOTH_VORTEX, CY_SIN3D, CY_DIV_TEST, CY_ORSZAG_TANG, CY_ORSZAG_TANG2, CY_EXPLOSION, CY_ROTOR, CY_JET = range(8)
CY_PROBLEMS = tuple(range(8))
CY_FLUX_CENTRAL, CY_FLUX_LF, CY_FLUX_HLL = 0, 1, 2


class GdfCyConfig(C.Structure):
    _fields_ = [
        ("nr", C.c_int32), ("nz", C.c_int32), ("lphi", C.c_int32),
        ("bc_r", C.c_int32), ("bc_l", C.c_int32), ("bc_u", C.c_int32), ("bc_d", C.c_int32),
        ("flux_type", C.c_int32), ("rhsc_open", C.c_int32), ("reserved_i", C.c_int32),
        ("ra", C.c_double), ("rb", C.c_double), ("za", C.c_double), ("zb", C.c_double),
        ("gamma", C.c_double), ("cfl", C.c_double), ("tvb_m", C.c_double), ("change_tol", C.c_double),
        ("jet_r", C.c_double), ("reserved_d", C.c_double * 3),
    ]

    def copy(self) -> "GdfCyConfig":
        out = GdfCyConfig()
        C.memmove(C.byref(out), C.byref(self), C.sizeof(GdfCyConfig))
        return out

    def as_dict(self) -> dict:
        return {name: (getattr(self, name) if name != "reserved_d" else list(self.reserved_d))
                for name, _ in self._fields_}


def cy_problem_config(problem: int, nr: int, nz: int, lphi: int = 1) -> tuple[GdfCyConfig, float]:
    """Pure-Python twin of gdf_cy_config_problem(): the domain, boundaries,
    M and switches of init0.txt .. init7.txt, with com.txt's constants
    (flux_type 2, gamma 5/3) and calculate_dt.f90:8's CFL 0.2."""
    pi = 4 * math.atan(1.0)
    c = GdfCyConfig()
    c.nr, c.nz, c.lphi = nr, nz, lphi
    c.flux_type = CY_FLUX_HLL
    c.gamma = 5.0 / 3.0
    c.cfl = 0.2
    c.change_tol = 1e-6
    c.jet_r = 1.5
    table = {
        CY_SMOOTH_VORTEX: ((-5.0, 5.0, -5.0, 5.0), (1, 1, 1, 1), 1.0, 1000000.0, 0),
        CY_SIN3D: ((2 * pi, 4 * pi, 0.0, 2 * pi), (4, 4, 1, 1), 1.0, 1000000.0, 1),
        CY_DIV_TEST: ((2 * pi, 4 * pi, 0.0, 2 * pi), (4, 4, 1, 1), 0.0, 1000000.0, 1),
        CY_ORSZAG_TANG: ((6 * pi, 8 * pi, 0.0, 2 * pi), (1, 1, 1, 1), 4.0, 10.0, 0),
        CY_ORSZAG_TANG2: ((10 * pi, 12 * pi, 0.0, 2 * pi), (4, 4, 1, 1), 0.5, 1.0, 0),
        CY_EXPLOSION: ((0.1, 1.0, -0.5, 0.5), (2, 2, 2, 2), 0.001, 1.0, 0),
        CY_ROTOR: ((1.0, 2.0, 0.0, 1.0), (2, 2, 2, 2), 0.015, 1.0, 0),
        CY_JET: ((1.0, 2.0, 0.0, 1.0), (5, 5, 2, 2), 0.6, 1000000.0, 0),
    }
    if problem not in table:
        raise ValueError(f"problem {problem} has no init file in MHD_GDF_cy3D_0421/")
    (c.ra, c.rb, c.za, c.zb), (c.bc_r, c.bc_l, c.bc_u, c.bc_d), tend, c.tvb_m, c.rhsc_open = table[problem]
    return c, tend


def cy_uh_shape(nr: int, nz: int, lphi: int) -> tuple:
    return (NE, NPC, 2 * lphi, nz + 2, nr + 2)


def cy_br_shape(nr: int, nz: int, lphi: int) -> tuple:
    return (3, 2 * lphi, nz, nr + 1)


def cy_bz_shape(nr: int, nz: int, lphi: int) -> tuple:
    return (3, 2 * lphi, nz + 1, nr)


def cy_new_state(nr: int, nz: int, lphi: int):
    return (np.zeros(cy_uh_shape(nr, nz, lphi)), np.zeros(cy_br_shape(nr, nz, lphi)),
            np.zeros(cy_bz_shape(nr, nz, lphi)))


def cy_live_mask() -> np.ndarray:
    """(8, 10) bool: the slots the method can make non-zero
    (div_free_Balsara.f90:125-143 writes the cubic modes of r*B)."""
    m = np.zeros((NE, NPC), bool)
    m[:, :NQC] = True
    m[5, 6:9] = True     # a30, a21, a12 (modes 7-9 of r*B_r)
    m[6, 7:10] = True    # b21, b12, b03 (modes 8-10 of r*B_z)
    return m


def _declare(L) -> None:
    if getattr(L, "_gdf_cy_declared", False):
        return
    vp, dp, i32 = C.c_void_p, C.POINTER(C.c_double), C.c_int32
    cp = C.POINTER(GdfCyConfig)
    L.gdf_cy_config_problem.argtypes = [i32, i32, i32, i32, cp, dp]
    L.gdf_cy_init_data.argtypes = [cp, i32, dp, dp, dp]
    L.gdf_cy_create.argtypes = [cp, C.POINTER(vp)]
    L.gdf_cy_destroy.argtypes = [vp]
    L.gdf_cy_upload.argtypes = [vp, dp, dp, dp]
    L.gdf_cy_download.argtypes = [vp, dp, dp, dp]
    L.gdf_cy_set_time.argtypes = [vp, C.c_double]
    L.gdf_cy_get_time.argtypes = [vp, dp]
    L.gdf_cy_prepare.argtypes = [vp]
    L.gdf_cy_step.argtypes = [vp, C.c_double, dp, dp]
    L.gdf_cy_advance.argtypes = [vp, C.c_double, i32, dp, C.POINTER(i32)]
    L.gdf_cy_advance_timed.argtypes = [vp, C.c_double, i32, dp, C.POINTER(i32), dp]
    L.gdf_cy_lh.argtypes = [vp, dp, dp, dp, C.c_double, dp, dp, dp]
    L.gdf_cy_limit.argtypes = [vp, dp, dp, dp]
    L.gdf_cy_dt.argtypes = [vp, dp, dp]
    L.gdf_cy_diagnostics.argtypes = [vp, dp, dp, dp]
    L.gdf_cy_kernel_launches.argtypes = [vp, C.POINTER(C.c_int64)]
    L._gdf_cy_declared = True


def _lib(exact: bool = True):
    from . import load
    L = load(exact)
    _declare(L)
    return L


def _check(L, rc: int) -> None:
    from . import _check as ck
    ck(L, rc)


def c_cy_problem_config(problem: int, nr: int, nz: int, lphi: int = 1, exact: bool = True):
    """gdf_cy_config_problem through the library."""
    L = _lib(exact)
    c = GdfCyConfig()
    tend = C.c_double()
    _check(L, L.gdf_cy_config_problem(problem, nr, nz, lphi, C.byref(c), C.byref(tend)))
    return c, tend.value


def cy_init_data(cfg: GdfCyConfig, problem: int, exact: bool = True):
    """gdf_cy_init_data: the host projection of the initial data."""
    L = _lib(exact)
    uh, br, bz = cy_new_state(cfg.nr, cfg.nz, cfg.lphi)
    _check(L, L.gdf_cy_init_data(C.byref(cfg), problem, dptr(uh), dptr(br), dptr(bz)))
    return uh, br, bz


class CySolver:
    """One device-resident cylindrical problem (a gdf_cy_create handle)."""

    def __init__(self, cfg: GdfCyConfig, exact: bool = True):
        self.L = _lib(exact)
        self.cfg = cfg.copy()
        self.nr, self.nz, self.lphi = cfg.nr, cfg.nz, cfg.lphi
        h = C.c_void_p()
        _check(self.L, self.L.gdf_cy_create(C.byref(self.cfg), C.byref(h)))
        self.h = h
        self.t = 0.0

    def close(self) -> None:
        if getattr(self, "h", None):
            self.L.gdf_cy_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, uh, br, bz) -> None:
        _check(self.L, self.L.gdf_cy_upload(self.h, dptr(uh), dptr(br), dptr(bz)))
        self.t = 0.0

    def download(self):
        uh, br, bz = cy_new_state(self.nr, self.nz, self.lphi)
        _check(self.L, self.L.gdf_cy_download(self.h, dptr(uh), dptr(br), dptr(bz)))
        return uh, br, bz

    def set_time(self, t: float) -> None:
        _check(self.L, self.L.gdf_cy_set_time(self.h, t))
        self.t = t

    def prepare(self) -> None:
        _check(self.L, self.L.gdf_cy_prepare(self.h))

    def step(self, tend: float):
        t = C.c_double()
        dt = C.c_double()
        _check(self.L, self.L.gdf_cy_step(self.h, tend, C.byref(t), C.byref(dt)))
        self.t = t.value
        return t.value, dt.value

    def advance(self, tend: float, max_steps: int):
        t = C.c_double()
        n = C.c_int32()
        _check(self.L, self.L.gdf_cy_advance(self.h, tend, max_steps, C.byref(t), C.byref(n)))
        self.t = t.value
        return t.value, n.value

    def advance_timed(self, tend: float, steps: int):
        """(t, steps taken, device ms) of `steps` graph replays."""
        t = C.c_double()
        n = C.c_int32()
        ms = C.c_double()
        _check(self.L, self.L.gdf_cy_advance_timed(self.h, tend, steps, C.byref(t), C.byref(n), C.byref(ms)))
        self.t = t.value
        return t.value, n.value, ms.value

    def kernel_launches(self) -> int:
        n = C.c_int64()
        _check(self.L, self.L.gdf_cy_kernel_launches(self.h, C.byref(n)))
        return int(n.value)

    def lh(self, uh, br, bz, t_rk: float = 0.0):
        """Lh and LhEz of the given state: (du, dbr, dbz)."""
        du, dbr, dbz = np.zeros_like(uh), np.zeros_like(br), np.zeros_like(bz)
        _check(self.L, self.L.gdf_cy_lh(self.h, dptr(uh), dptr(br), dptr(bz), t_rk, dptr(du), dptr(dbr),
                                        dptr(dbz)))
        return du, dbr, dbz

    def limit(self, uh, br, bz) -> None:
        """TVB_Limiter_P2 then div_free_Balsara, in place."""
        _check(self.L, self.L.gdf_cy_limit(self.h, dptr(uh), dptr(br), dptr(bz)))

    def dt(self, uh) -> float:
        d = C.c_double()
        _check(self.L, self.L.gdf_cy_dt(self.h, dptr(uh), C.byref(d)))
        return d.value

    def diagnostics(self):
        a, b, p = C.c_double(), C.c_double(), C.c_double()
        _check(self.L, self.L.gdf_cy_diagnostics(self.h, C.byref(a), C.byref(b), C.byref(p)))
        return a.value, b.value, p.value
