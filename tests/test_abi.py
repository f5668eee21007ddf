"""The C-ABI library: symbols, struct layout, host-only entry points.

No compute call here needs a GPU: gdf_config_reference, gdf_problem_config
and gdf_init_data are host code (the reference's L0/L1 set-up)."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import gdf
from gdf import _abi
from oracle import Oracle

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "gdf.h")
PROBLEMS = [gdf.PROB_VORTEX, gdf.PROB_ORSZAG_TANG, gdf.PROB_ROTOR, gdf.PROB_BLAST, gdf.PROB_CLOUD_SHOCK]


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gdf_[a-z_0-9]+)\s*\(", src)))


@pytest.mark.parametrize("exact", [False, True])
def test_every_declared_symbol_is_exported(exact):
    lib = gdf.LIB_EXACT if exact else gdf.LIB_FMA
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (gdf_\w+)", out))
    syms = declared_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if s not in exported]
    assert not missing, f"declared in gdf.h but not exported: {missing}"
    L = gdf.load(exact)
    for s in syms:
        assert hasattr(L, s)
    assert L.gdf_build_exact() == (1 if exact else 0)


def test_config_struct_layout_matches_c(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text('#include <stddef.h>\n#include "gdf.h"\n'
                   "size_t cfg_size(void){return sizeof(GdfConfig);}\n"
                   "size_t off_ck(void){return offsetof(GdfConfig, kxrcf_ck);}\n"
                   "size_t off_res(void){return offsetof(GdfConfig, reserved_d);}\n")
    so = tmp_path / "libsz.so"
    subprocess.run(["gcc", "-shared", "-fPIC", "-I", os.path.join(REPO, "include"), "-o", str(so), str(src)],
                   check=True)
    L = C.CDLL(str(so))
    for f in ("cfg_size", "off_ck", "off_res"):
        getattr(L, f).restype = C.c_size_t
    assert L.cfg_size() == C.sizeof(_abi.GdfConfig)
    assert L.off_ck() == _abi.GdfConfig.kxrcf_ck.offset
    assert L.off_res() == _abi.GdfConfig.reserved_d.offset


@pytest.mark.parametrize("problem", PROBLEMS)
def test_problem_config_python_twin_matches_c(problem):
    c_cfg, c_tend = gdf.c_problem_config(problem, 24, 16)
    p_cfg, p_tend = gdf.problem_config(problem, 24, 16)
    assert c_tend == p_tend
    assert c_cfg.as_dict() == p_cfg.as_dict()


def test_reference_config_matches_c():
    L = gdf.load()
    c = gdf.GdfConfig()
    assert L.gdf_config_reference(80, 40, C.byref(c)) == 0
    assert c.as_dict() == gdf.reference_config(80, 40).as_dict()


@pytest.mark.parametrize("problem", PROBLEMS)
def test_init_data_matches_oracle_bitwise(problem):
    cfg, _ = gdf.problem_config(problem, 12, 10)
    uh, bx, by = gdf.init_data(cfg, problem)
    o = Oracle(cfg)
    uh2, bx2, by2 = o.init_data(problem)
    assert np.array_equal(uh, uh2)
    assert np.array_equal(bx, bx2)
    assert np.array_equal(by, by2)


def test_init_data_rejects_bad_arguments():
    L = gdf.load()
    cfg, _ = gdf.problem_config(gdf.PROB_ORSZAG_TANG, 4, 4)
    uh, bx, by = gdf.new_state(4, 4)
    assert L.gdf_init_data(C.byref(cfg), 9, None, _abi.dptr(uh), _abi.dptr(bx), _abi.dptr(by)) == gdf._abi.GDF_ERR_ARG
    assert L.gdf_problem_config(7, 4, 4, C.byref(cfg), None) == gdf._abi.GDF_ERR_ARG


def test_create_without_device_fails_loudly(has_gpu):
    if has_gpu:
        pytest.skip("a device is present")
    cfg, _ = gdf.problem_config(gdf.PROB_ORSZAG_TANG, 8, 8)
    with pytest.raises(gdf.GdfError) as e:
        gdf.Solver(cfg)
    assert e.value.code == gdf._abi.GDF_ERR_CUDA
