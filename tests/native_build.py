"""Host build of tests/native/devcheck.cpp: the library's pointwise physics
header compiled for the CPU without FMA, for value-exact comparison with the
oracle."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "native", "_build")
LIB = os.path.join(OUT_DIR, "libdevcheck.so")
SRC = os.path.join(HERE, "native", "devcheck.cpp")
HDR = os.path.join(os.path.dirname(HERE), "freljord-cfd-arsenal_b200", "csrc", "gdf_physics.cuh")
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def build_devcheck() -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    if (not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(SRC), os.path.getmtime(HDR))):
        subprocess.run([CXX, "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-march=x86-64",
                        "-Wno-unknown-pragmas", "-o", LIB, SRC], check=True)
    return LIB
