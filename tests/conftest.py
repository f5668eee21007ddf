"""Shared fixtures: paths to the library and the oracle, the `gpu` marker,
and a session-level build of everything the tests load."""
import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "freljord-cfd-arsenal_b200")
for p in (PKG, os.path.join(REPO, "oracle"), os.path.join(REPO, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def _build_all():
    import build as pkg_build  # freljord-cfd-arsenal_b200/build.py
    pkg_build.build()
    subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle")], check=True)
    from native_build import build_devcheck
    build_devcheck()


@pytest.fixture(scope="session", autouse=True)
def built():
    _build_all()
    return True


@pytest.fixture(scope="session")
def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
