"""Build the sm_100a shared libraries of the GDF P2 step, in-tree.

Produces, under freljord-cfd-arsenal_b200/lib/:
  libgdf_b200.so        the product build: --fmad=false, so every FP64
                        operation rounds as in an FMA-free CPU build of the
                        reference (bit-faithful step, identical flag sets)
  libgdf_b200_fma.so    the same sources with FMA contraction on (faster
                        arithmetic; results differ in the last bits and can
                        flip a limiter decision that sits on a threshold)
Both export the C ABI of include/gdf.h. Rebuilds only what is out of date.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "lib")
BUILD = os.path.join(PKG, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
HOST_CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"

KERNEL_SRC = os.path.join(CSRC, "gdf_kernels.cu")
MLP_SRC = os.path.join(CSRC, "gdf_mlp.cu")
ENS_SRC = os.path.join(CSRC, "gdf_ensemble.cu")
PEAK_SRC = os.path.join(CSRC, "gdf_peak.cu")
INIT_SRC = os.path.join(CSRC, "gdf_init.cu")
MLPTC_SRC = os.path.join(CSRC, "gdf_mlp_tc.cu")
P3_SRC = os.path.join(CSRC, "gdf_p3.cu")
CY_SRC = os.path.join(CSRC, "gdf_cy.cu")
HOST_SRC = os.path.join(CSRC, "gdf_host.cpp")
IO_SRC = os.path.join(CSRC, "gdf_io.cpp")
CYHOST_SRC = os.path.join(CSRC, "gdf_cy_host.cpp")
HEADERS = [os.path.join(CSRC, f) for f in ("gdf_physics.cuh", "gdf_kernels.cuh", "gdf_device.cuh",
                                                         "gdf_mlp.cuh", "gdf_p3_basis.h")] + [
    os.path.join(REPO, "include", "gdf.h"), os.path.join(REPO, "include", "gdf_p3.h"),
    os.path.join(REPO, "include", "gdf_cy.h")]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build the library")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build failed: " + " ".join(cmd[:3]) + " ...")


def build(verbose: bool = False, jobs: int | None = None) -> dict:
    """Compile what is stale; the CUDA objects of both libraries compile
    concurrently (`jobs` at a time, default: the host's cores, at most 6)."""
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(LIB, exist_ok=True)
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    host_o = os.path.join(BUILD, "gdf_host.o")
    io_o = os.path.join(BUILD, "gdf_io.o")
    cyh_o = os.path.join(BUILD, "gdf_cy_host.o")
    cmds = []
    for src, obj in ((HOST_SRC, host_o), (IO_SRC, io_o), (CYHOST_SRC, cyh_o)):
        if _stale(obj, [src] + HEADERS):
            cmds.append([HOST_CXX, "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-march=x86-64", "-fopenmp",
                         "-c", src, "-o", obj])
    libs = []
    for name, flags in (("libgdf_b200.so", ["--fmad=false", "-DGDF_EXACT=1"]),
                        ("libgdf_b200_fma.so", ["--fmad=true"])):
        objs = []
        for src in (KERNEL_SRC, MLP_SRC, ENS_SRC, PEAK_SRC, INIT_SRC, MLPTC_SRC, P3_SRC, CY_SRC):
            obj = os.path.join(BUILD, name.replace(".so", "") + "_" + os.path.basename(src).replace(".cu", ".o"))
            if _stale(obj, [src] + HEADERS):
                cmd = [nvcc, *ARCH, "-lineinfo", "-O3", "-std=c++17", *flags,
                       "-Xcompiler", "-fPIC,-ffp-contract=off", "-c", src, "-o", obj]
                if verbose:
                    cmd.insert(1, "-Xptxas=-v")
                cmds.append(cmd)
            objs.append(obj)
        libs.append((name, objs))
    if cmds:
        n = jobs or max(1, min(6, os.cpu_count() or 1))
        with ThreadPoolExecutor(max_workers=n) as ex:
            for f in [ex.submit(_run, c) for c in cmds]:
                f.result()
    out = {}
    for name, objs in libs:
        so = os.path.join(LIB, name)
        if _stale(so, objs + [host_o, io_o, cyh_o]):
            _run([nvcc, *ARCH, "-shared", "-o", so, *objs, host_o, io_o, cyh_o, "-Xcompiler", "-fopenmp", "-lgomp"])
        out[name] = so
    return out


if __name__ == "__main__":
    for k, v in build(verbose="-v" in sys.argv).items():
        print(k, "->", v)
