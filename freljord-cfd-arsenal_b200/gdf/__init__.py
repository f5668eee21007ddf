"""Python host mirror of the reference's driver (main.f90 / RK3.f90) over the
C ABI of include/gdf.h, for the B200 GDF P2 solver.

The solver itself is the sm_100a library ``lib/libgdf_b200.so`` (built
without FMA contraction, so its arithmetic follows the reference's) or, on
request, ``lib/libgdf_b200_fma.so`` (FMA contraction on); this module only
binds it with ctypes. There is no CPU fallback: if the library is missing or no
CUDA device is present, the constructors raise.

Mapping to the reference (paths relative to GDF_Balsara_P2_0316/):
  problem_config / init_data   init_data.f90 with an init*.txt problem
  Solver.prepare               RK3.f90:5-12 (set_bc, TVB_Limiter_P2, div_free)
  Solver.step                  one pass of the RK3.f90:58-174 loop body
  Solver.advance               the RK3.f90 loop (device resident, graph)
  Solver.lh / lhez / limit / dt  Lh, LhEz, TVB_Limiter_P2 + div_free_Balsara,
                                 calculate_dt on caller arrays
  Solver.diagnostics           calculate_umax / _totaldiv / _pmin
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from ._abi import (BC_OUTFLOW, BC_PERIODIC, DETECT_ALL, DETECT_KXRCF, FLUX_HLL, FLUX_HLLC, FLUX_HLLD,  # noqa: F401
                   FLUX_LF, GDF_OK, LIB_DIR, NE, NP, PROB_BLAST, PROB_CLOUD_SHOCK, PROB_ORSZAG_TANG,
                   PROB_ROTOR, PROB_VORTEX, GdfConfig, bx_shape, by_shape, dptr, iptr, new_state,
                   problem_config, reference_config, uh_shape)

DETECT_LEARNED = 2
ENS_TUNE_CANDIDATES = 45
MLP_NPARAM = 10049
NFEAT = 90

KERNEL_NAMES = ["set_bc", "face_x", "face_y", "vertex", "cell", "bface", "limit", "dt", "diag", "faceb_limit",
                "divfree", "limit_tvb"]
KERNEL_KINDS = len(KERNEL_NAMES)

LIB_EXACT = os.path.join(LIB_DIR, "libgdf_b200.so")
LIB_FMA = os.path.join(LIB_DIR, "libgdf_b200_fma.so")
LIB_FAST = LIB_FMA

_libs: dict = {}


class GdfError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"gdf error {code}: {msg}")
        self.code = code


def load(exact: bool = True):
    """Load the sm_100a library (the product build, or the FMA build when
    exact is False) and declare the ABI."""
    path = LIB_EXACT if exact else LIB_FMA
    if path in _libs:
        return _libs[path]
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with freljord-cfd-arsenal_b200/build.py "
                          "(the solver has no CPU fallback)")
    L = C.CDLL(path)
    vp, dp, ip, i32 = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int32), C.c_int32
    cfgp = C.POINTER(GdfConfig)
    L.gdf_last_error.restype = C.c_char_p
    L.gdf_build_exact.restype = C.c_int
    L.gdf_config_reference.argtypes = [i32, i32, cfgp]
    L.gdf_problem_config.argtypes = [i32, i32, i32, cfgp, dp]
    L.gdf_init_data.argtypes = [cfgp, i32, dp, dp, dp, dp]
    L.gdf_create.argtypes = [cfgp, C.POINTER(vp)]
    L.gdf_destroy.argtypes = [vp]
    L.gdf_upload.argtypes = [vp, dp, dp, dp]
    L.gdf_download.argtypes = [vp, dp, dp, dp]
    L.gdf_download_live.argtypes = [vp, dp, dp, dp]
    L.gdf_upload_state.argtypes = [vp, dp, dp, dp]
    L.gdf_download_state.argtypes = [vp, dp, dp, dp]
    L.gdf_prepare.argtypes = [vp, ip]
    L.gdf_step.argtypes = [vp, C.c_double, dp, dp, ip]
    L.gdf_advance.argtypes = [vp, C.c_double, i32, dp, ip]
    L.gdf_lh.argtypes = [vp, dp, dp]
    L.gdf_lhez.argtypes = [vp, dp, dp, dp]
    L.gdf_limit.argtypes = [vp, dp, dp, dp, ip]
    L.gdf_dt.argtypes = [vp, dp, dp]
    L.gdf_diagnostics.argtypes = [vp, dp, dp, dp, C.POINTER(C.c_int64)]
    L.gdf_get_time.argtypes = [vp, dp, dp]
    L.gdf_set_time.argtypes = [vp, C.c_double]
    L.gdf_kernel_launches.argtypes = [vp]
    L.gdf_kernel_launches.restype = C.c_int64
    L.gdf_stream.argtypes = [vp]
    L.gdf_stream.restype = C.c_void_p
    L.gdf_profile.argtypes = [vp, i32, dp, C.POINTER(C.c_int64), i32]
    L.gdf_advance_timed.argtypes = [vp, C.c_double, i32, dp, ip, dp]
    L.gdf_set_device.argtypes = [i32]
    L.gdf_lh_noalloc.argtypes = [cfgp, vp, vp, vp]
    L.gdf_fp64_fma_peak.argtypes = [i32, i32, dp, dp]
    L.gdf_init_data_device.argtypes = [vp, i32, dp]
    cp = C.c_char_p
    L.gdf_save_solution.argtypes = [cfgp, dp, cp]
    L.gdf_save_frame.argtypes = [cfgp, dp, C.c_double, cp, i32]
    L.gdf_save_xy.argtypes = [cfgp, cp]
    L.gdf_l2_error.argtypes = [cfgp, dp, C.c_double, dp]
    L.gdf_config_of.argtypes = [vp, cfgp]
    L.gdf_get_trouble.argtypes = [vp, ip]
    L.gdf_set_trouble.argtypes = [vp, ip]
    L.gdf_checkpoint_save.argtypes = [vp, cp]
    L.gdf_checkpoint_load.argtypes = [vp, cp]
    fp = C.POINTER(C.c_float)
    L.gdf_features.argtypes = [vp, dp, fp]
    L.gdf_mlp_create.argtypes = [i32, C.POINTER(vp)]
    L.gdf_mlp_destroy.argtypes = [vp]
    L.gdf_mlp_set_params.argtypes = [vp, fp]
    L.gdf_mlp_get_params.argtypes = [vp, fp]
    L.gdf_mlp_grad.argtypes = [vp, fp, fp, C.c_int64, C.c_float, fp, fp]
    L.gdf_mlp_train.argtypes = [vp, fp, fp, C.c_int64, i32, i32, C.c_float, C.c_float, i32, fp]
    L.gdf_mlp_predict.argtypes = [vp, fp, C.c_int64, fp]
    L.gdf_mlp_last_error.restype = C.c_char_p
    L.gdf_mlp_set_products.argtypes = [vp, i32]
    L.gdf_set_indicator.argtypes = [vp, vp, C.c_float, C.c_float]
    L.gdf_ens_create.argtypes = [cfgp, i32, C.POINTER(vp)]
    L.gdf_ens_destroy.argtypes = [vp]
    L.gdf_ens_upload.argtypes = [vp, i32, dp, dp, dp]
    L.gdf_ens_download.argtypes = [vp, i32, dp, dp, dp]
    L.gdf_ens_set_indicator.argtypes = [vp, vp, C.c_float, C.c_float]
    L.gdf_ens_set_time.argtypes = [vp, i32, C.c_double, C.c_double]
    L.gdf_ens_get_time.argtypes = [vp, i32, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int64)]
    L.gdf_ens_prepare.argtypes = [vp]
    L.gdf_ens_advance.argtypes = [vp, i32, C.POINTER(C.c_int64), C.POINTER(i32), C.POINTER(C.c_double)]
    L.gdf_ens_set_tiles.argtypes = [vp, i32, i32, i32]
    L.gdf_ens_get_tiles.argtypes = [vp] + [C.POINTER(i32)] * 6
    L.gdf_ens_set_mode.argtypes = [vp, i32]
    L.gdf_ens_tune.argtypes = [vp, i32, C.POINTER(C.c_float)]
    L.gdf_ens_kernel_launches.argtypes = [vp]
    L.gdf_ens_barrier_selftest.argtypes = [i32, i32, C.c_uint64, ip]
    L.gdf_ens_kernel_launches.restype = C.c_int64
    L.gdf_ens_last_error.restype = C.c_char_p
    _libs[path] = L
    return L


def _check(L, rc: int) -> None:
    if rc != GDF_OK:
        raise GdfError(rc, L.gdf_last_error().decode())


def set_device(device: int, exact: bool = True) -> None:
    """gdf_set_device: the CUDA device this library uses on this thread."""
    L = load(exact)
    _check(L, L.gdf_set_device(device))


def lh_noalloc(cfg: GdfConfig, d_uh: int, d_du: int, stream: int = 0, exact: bool = True) -> None:
    """gdf_lh_noalloc: Lh on caller-owned device buffers (device pointers as
    integers), enqueued on `stream`; allocates no device memory."""
    L = load(exact)
    _check(L, L.gdf_lh_noalloc(C.byref(cfg), C.c_void_p(d_uh), C.c_void_p(d_du), C.c_void_p(stream or None)))


def fp64_fma_peak(blocks_per_sm: int = 4, iters: int = 20000, exact: bool = True):
    """gdf_fp64_fma_peak: (TFLOP/s, ms) of an FMA-only kernel on every SM of
    the current device, timed with CUDA events."""
    L = load(exact)
    tf, ms = C.c_double(), C.c_double()
    _check(L, L.gdf_fp64_fma_peak(blocks_per_sm, iters, C.byref(tf), C.byref(ms)))
    return tf.value, ms.value


def c_problem_config(problem: int, nx: int, ny: int, exact: bool = True):
    """gdf_problem_config through the library (host-only call)."""
    L = load(exact)
    cfg = GdfConfig()
    te = C.c_double()
    _check(L, L.gdf_problem_config(problem, nx, ny, C.byref(cfg), C.byref(te)))
    return cfg, te.value


def init_data(cfg: GdfConfig, problem: int, params=None, exact: bool = True):
    """init_data.f90 on the host: returns (uh, bx, by) in the reference layout."""
    L = load(exact)
    uh, bx, by = new_state(cfg.nx, cfg.ny)
    p = None if params is None else dptr(np.ascontiguousarray(params, np.float64))
    _check(L, L.gdf_init_data(C.byref(cfg), problem, p, dptr(uh), dptr(bx), dptr(by)))
    return uh, bx, by


def save_solution(cfg: GdfConfig, uh, directory: str = ".", exact: bool = True) -> None:
    """save_solution.f90: Q1.txt..Q8.txt of uh in directory."""
    L = load(exact)
    _check(L, L.gdf_save_solution(C.byref(cfg), dptr(uh), directory.encode()))


def save_frame(cfg: GdfConfig, uh, t: float, directory: str = ".", reset: bool = False,
               exact: bool = True) -> None:
    """One frame of RK3.f90's Q*flash.txt / T.txt output (reset: new files)."""
    L = load(exact)
    _check(L, L.gdf_save_frame(C.byref(cfg), dptr(uh), t, directory.encode(), 1 if reset else 0))


def save_xy(cfg: GdfConfig, directory: str = ".", exact: bool = True) -> None:
    """save_XY.f90: Xc.txt, Yc.txt, lambda.txt, weight.txt."""
    L = load(exact)
    _check(L, L.gdf_save_xy(C.byref(cfg), directory.encode()))


def l2_error(cfg: GdfConfig, uh, t20: float = 0.0, exact: bool = True) -> np.ndarray:
    """calculate_L2error.f90 against the vortex of init1.txt moved by (t20, t20)."""
    L = load(exact)
    out = np.zeros(NE)
    _check(L, L.gdf_l2_error(C.byref(cfg), dptr(uh), t20, dptr(out)))
    return out


class Solver:
    """One device-resident GDF P2 problem (a gdf_create handle)."""

    def __init__(self, cfg: GdfConfig, exact: bool = True):
        self.L = load(exact)
        self.cfg = cfg.copy()
        self.nx, self.ny = cfg.nx, cfg.ny
        h = C.c_void_p()
        _check(self.L, self.L.gdf_create(C.byref(self.cfg), C.byref(h)))
        self.h = h
        self.t = 0.0

    def close(self) -> None:
        if getattr(self, "h", None):
            self.L.gdf_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _flags(self):
        return np.zeros((self.ny, self.nx), np.int32)

    def upload(self, uh, bx, by) -> None:
        _check(self.L, self.L.gdf_upload(self.h, dptr(uh), dptr(bx), dptr(by)))

    def init_device(self, problem: int, params=None) -> None:
        """gdf_init_data_device: the problem's initial data projected on the
        device into the resident state (no host state, no upload)."""
        p = None if params is None else dptr(np.ascontiguousarray(params, np.float64))
        _check(self.L, self.L.gdf_init_data_device(self.h, problem, p))

    def download(self):
        uh, bx, by = new_state(self.nx, self.ny)
        _check(self.L, self.L.gdf_download(self.h, dptr(uh), dptr(bx), dptr(by)))
        return uh, bx, by

    def features(self, uh):
        """gdf_features: the indicator's 90 inputs per interior cell."""
        X = np.zeros((self.nx * self.ny, NFEAT), np.float32)
        _check(self.L, self.L.gdf_features(self.h, dptr(uh), X.ctypes.data_as(C.POINTER(C.c_float))))
        return X

    def set_indicator(self, mlp: "Mlp", t_lo: float = 0.5, t_hi: float = 0.5) -> None:
        _check(self.L, self.L.gdf_set_indicator(self.h, mlp.h, t_lo, t_hi))

    def download_into(self, uh, bx, by, live_only: bool = False) -> None:
        """gdf_download into caller arrays (e.g. pinned host buffers);
        live_only: gdf_download_live (dead slot planes of uh not written)."""
        f = self.L.gdf_download_live if live_only else self.L.gdf_download
        _check(self.L, f(self.h, dptr(uh), dptr(bx), dptr(by)))

    def state_shape(self) -> tuple:
        """numpy shape (v, d, j, i) of the compact step state of
        gdf_upload_state / gdf_download_state: modes 1-6 of variables
        1-5 and 8 over the interior cells."""
        return (6, 6, self.ny, self.nx)

    def upload_state(self, cells, bx, by) -> None:
        """gdf_upload_state: the compact state; the device rebuilds the cell
        B modes (div-free reconstruction) and the ghosts (set_bc)."""
        _check(self.L, self.L.gdf_upload_state(self.h, dptr(cells), dptr(bx), dptr(by)))

    def download_state(self, cells=None, bx=None, by=None):
        """gdf_download_state into caller arrays (allocated when None)."""
        if cells is None:
            cells = np.zeros(self.state_shape())
        if bx is None or by is None:
            _, bx, by = new_state(self.nx, self.ny)
        _check(self.L, self.L.gdf_download_state(self.h, dptr(cells), dptr(bx), dptr(by)))
        return cells, bx, by

    def prepare(self):
        f = self._flags()
        _check(self.L, self.L.gdf_prepare(self.h, iptr(f)))
        self.t = 0.0
        return f

    def step(self, tend: float, flags: bool = True):
        t = C.c_double(self.t)
        dt = C.c_double()
        f = self._flags() if flags else None
        _check(self.L, self.L.gdf_step(self.h, tend, C.byref(t), C.byref(dt), iptr(f) if flags else None))
        self.t = t.value
        return t.value, dt.value, f

    def advance(self, tend: float, max_steps: int):
        t = C.c_double(self.t)
        n = C.c_int32()
        _check(self.L, self.L.gdf_advance(self.h, tend, max_steps, C.byref(t), C.byref(n)))
        self.t = t.value
        return t.value, n.value

    def advance_timed(self, tend: float, steps: int):
        """(t, steps taken, device ms) of `steps` graph replays."""
        t = C.c_double(self.t)
        n = C.c_int32()
        ms = C.c_double()
        _check(self.L, self.L.gdf_advance_timed(self.h, tend, steps, C.byref(t), C.byref(n), C.byref(ms)))
        self.t = t.value
        return t.value, n.value, ms.value

    def lh(self, uh):
        du = np.zeros_like(uh)
        _check(self.L, self.L.gdf_lh(self.h, dptr(uh), dptr(du)))
        return du

    def lhez(self, uh):
        _, d1, d2 = new_state(self.nx, self.ny)
        _check(self.L, self.L.gdf_lhez(self.h, dptr(uh), dptr(d1), dptr(d2)))
        return d1, d2

    def limit(self, uh, bx, by):
        f = self._flags()
        _check(self.L, self.L.gdf_limit(self.h, dptr(uh), dptr(bx), dptr(by), iptr(f)))
        return f

    def dt(self, uh) -> float:
        d = C.c_double()
        _check(self.L, self.L.gdf_dt(self.h, dptr(uh), C.byref(d)))
        return d.value

    def diagnostics(self):
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        n = C.c_int64()
        _check(self.L, self.L.gdf_diagnostics(self.h, C.byref(a), C.byref(b), C.byref(c), C.byref(n)))
        return a.value, b.value, c.value, n.value

    def time(self):
        t, dt = C.c_double(), C.c_double()
        _check(self.L, self.L.gdf_get_time(self.h, C.byref(t), C.byref(dt)))
        return t.value, dt.value

    def set_time(self, t: float) -> None:
        _check(self.L, self.L.gdf_set_time(self.h, t))
        self.t = t

    def kernel_launches(self) -> int:
        return self.L.gdf_kernel_launches(self.h)

    def trouble(self):
        """The sticky KXRCF flags (Is_Trouble_Cell), shape (ny, nx)."""
        f = self._flags()
        _check(self.L, self.L.gdf_get_trouble(self.h, iptr(f)))
        return f

    def set_trouble(self, f) -> None:
        f = np.ascontiguousarray(f, np.int32)
        _check(self.L, self.L.gdf_set_trouble(self.h, iptr(f)))

    def checkpoint(self, path: str) -> None:
        """gdf_checkpoint_save: state, time and sticky flags to a file."""
        _check(self.L, self.L.gdf_checkpoint_save(self.h, os.fsencode(path)))

    def restore(self, path: str) -> None:
        """gdf_checkpoint_load into this handle (same configuration)."""
        _check(self.L, self.L.gdf_checkpoint_load(self.h, os.fsencode(path)))
        self.t = self.time()[0]

    def stream(self) -> int:
        """The handle's cudaStream_t as an integer."""
        return self.L.gdf_stream(self.h) or 0

    def profile(self, steps: int = 1):
        """Per kernel kind: (mean ms per launch, launches per step)."""
        ms = np.zeros(KERNEL_KINDS)
        n = np.zeros(KERNEL_KINDS, np.int64)
        _check(self.L, self.L.gdf_profile(self.h, steps, dptr(ms), n.ctypes.data_as(C.POINTER(C.c_int64)),
                                          KERNEL_KINDS))
        return {KERNEL_NAMES[k]: (ms[k], int(n[k])) for k in range(KERNEL_KINDS)}


def _fptr(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_float))


class Mlp:
    """The learned troubled-cell indicator (90-64-64-1), trained and run by
    the library's tensor-core kernels."""

    def __init__(self, seed: int = 0, exact: bool = True):
        self.L = load(exact)
        h = C.c_void_p()
        rc = self.L.gdf_mlp_create(seed, C.byref(h))
        if rc:
            raise GdfError(rc, self.L.gdf_mlp_last_error().decode())
        self.h = h

    def _ck(self, rc):
        if rc:
            raise GdfError(rc, self.L.gdf_mlp_last_error().decode())

    def close(self):
        if getattr(self, "h", None):
            self.L.gdf_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_products(self, tcgen05: bool) -> None:
        """gdf_mlp_set_products: training products on tcgen05 (True, the
        default) or mma.sync (False)."""
        self._ck(self.L.gdf_mlp_set_products(self.h, 1 if tcgen05 else 0))

    def params(self) -> np.ndarray:
        p = np.zeros(MLP_NPARAM, np.float32)
        self._ck(self.L.gdf_mlp_get_params(self.h, _fptr(p)))
        return p

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == MLP_NPARAM
        self._ck(self.L.gdf_mlp_set_params(self.h, _fptr(p)))

    def grad(self, X, y, pos_weight: float = 1.0):
        X = np.ascontiguousarray(X, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        g = np.zeros(MLP_NPARAM, np.float32)
        loss = np.zeros(1, np.float32)
        self._ck(self.L.gdf_mlp_grad(self.h, _fptr(X), _fptr(y), len(y), pos_weight, _fptr(g), _fptr(loss)))
        return g, float(loss[0])

    def train(self, X, y, epochs: int = 10, batch: int = 1024, lr: float = 1e-3, pos_weight: float = 1.0,
              seed: int = 0):
        X = np.ascontiguousarray(X, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        losses = np.zeros(epochs, np.float32)
        self._ck(self.L.gdf_mlp_train(self.h, _fptr(X), _fptr(y), len(y), epochs, batch, lr, pos_weight, seed,
                                      _fptr(losses)))
        return losses

    def predict(self, X):
        X = np.ascontiguousarray(X, np.float32)
        p = np.zeros(len(X), np.float32)
        self._ck(self.L.gdf_mlp_predict(self.h, _fptr(X), len(X), _fptr(p)))
        return p


class Ensemble:
    """Independent problems of different sizes advanced together (the
    gdf_ens_* functions): one persistent kernel per RK stage, per-instance
    dt and end time."""

    def __init__(self, cfgs, exact: bool = True):
        self.L = load(exact)
        self.cfgs = [c.copy() for c in cfgs]
        arr = (GdfConfig * len(self.cfgs))(*self.cfgs)
        h = C.c_void_p()
        self._ck(self.L.gdf_ens_create(arr, len(self.cfgs), C.byref(h)))
        self.h = h
        self.n = len(self.cfgs)

    def _ck(self, rc):
        if rc:
            raise GdfError(rc, self.L.gdf_ens_last_error().decode())

    def close(self):
        if getattr(self, "h", None):
            self.L.gdf_ens_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, i: int, uh, bx, by) -> None:
        self._ck(self.L.gdf_ens_upload(self.h, i, dptr(uh), dptr(bx), dptr(by)))

    def download(self, i: int):
        c = self.cfgs[i]
        uh, bx, by = new_state(c.nx, c.ny)
        self._ck(self.L.gdf_ens_download(self.h, i, dptr(uh), dptr(bx), dptr(by)))
        return uh, bx, by

    def set_indicator(self, mlp: "Mlp", t_lo: float = 0.5, t_hi: float = 0.5) -> None:
        self._ck(self.L.gdf_ens_set_indicator(self.h, mlp.h, t_lo, t_hi))

    def set_time(self, i: int, t: float, tend: float) -> None:
        """t and tend of instance i (i = -1: every instance)."""
        self._ck(self.L.gdf_ens_set_time(self.h, i, t, tend))

    def time(self, i: int):
        t, dt, n = C.c_double(), C.c_double(), C.c_int64()
        self._ck(self.L.gdf_ens_get_time(self.h, i, C.byref(t), C.byref(dt), C.byref(n)))
        return t.value, dt.value, n.value

    def prepare(self) -> None:
        self._ck(self.L.gdf_ens_prepare(self.h))

    def advance(self, steps: int):
        """(cell updates, instances still running, device ms) of `steps`
        ensemble steps."""
        cu, na, ms = C.c_int64(), C.c_int32(), C.c_double()
        self._ck(self.L.gdf_ens_advance(self.h, steps, C.byref(cu), C.byref(na), C.byref(ms)))
        return cu.value, na.value, ms.value

    def set_tiles(self, ctas_per_sm: int = 0, face_per_thread: int = 1, cell_per_thread: int = 1) -> None:
        self._ck(self.L.gdf_ens_set_tiles(self.h, ctas_per_sm, face_per_thread, cell_per_thread))

    def set_mode(self, mode: int) -> None:
        """0: one persistent kernel per RK stage; 1: one launch per phase."""
        self._ck(self.L.gdf_ens_set_mode(self.h, mode))

    def tiles(self) -> dict:
        v = [C.c_int32() for _ in range(6)]
        self._ck(self.L.gdf_ens_get_tiles(self.h, *[C.byref(x) for x in v]))
        return dict(zip(["ctas_per_sm", "face_per_thread", "cell_per_thread", "grid", "graph", "mode"],
                        [x.value for x in v]))

    def tune(self, steps: int = 2):
        ms = np.zeros(ENS_TUNE_CANDIDATES, np.float32)
        self._ck(self.L.gdf_ens_tune(self.h, steps, _fptr(ms)))
        return ms

    def kernel_launches(self) -> int:
        return self.L.gdf_ens_kernel_launches(self.h)


def ensemble_configs(n: int = 64, seed: int = 0, detector: int = DETECT_LEARNED):
    """The ensemble workload: instance s takes, from a generator seeded by
    (seed, s), a problem in {Orszag-Tang, rotor, blast} and a square grid side
    in {64, 96, ..., 512}; all HLLD with the face-B minmod of the DF variants
    (without it the rotor at 288^2 loses positivity at step 6, the reference
    method's behaviour), the given detector (KXRCF fallback when learned).
    Returns [(config, problem, init params or None, tend)]."""
    out = []
    for s in range(n):
        rng = np.random.default_rng([seed, s])
        prob = [PROB_ORSZAG_TANG, PROB_ROTOR, PROB_BLAST][int(rng.integers(3))]
        side = 64 + 32 * int(rng.integers(15))
        cfg, tend = problem_config(prob, side, side)
        cfg.flux_type = FLUX_HLLD
        cfg.faceb_limiter = 1     # face-B minmod on every instance (see the blast and rotor notes)
        cfg.detector = detector
        if detector != DETECT_ALL:
            cfg.kxrcf_ck = 1.0
        params = None
        if prob == PROB_BLAST:
            from .indicator import blast_params
            params = blast_params(10_000 + 97 * seed + s)
        out.append((cfg, prob, params, tend))
    return out


def ens_barrier_selftest(blocks: int, skip_block: int, limit_ns: int, exact: bool = True) -> bool:
    """gdf_ens_barrier_selftest: True when the bounded barrier timed out."""
    L = load(exact)
    out = C.c_int32()
    rc = L.gdf_ens_barrier_selftest(blocks, skip_block, limit_ns, C.byref(out))
    if rc:
        raise GdfError(rc, L.gdf_ens_last_error().decode())
    return bool(out.value)
