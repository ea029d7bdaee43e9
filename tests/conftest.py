import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA library")


def _gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _gpu_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session", autouse=True)
def built_libraries():
    """Build (or reuse) the product library and the oracle once per session."""
    from piks3d_b200 import build as pbuild
    pbuild.build()
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    yield


def base_params(n, **kw):
    import piks3d_b200 as pk
    d = dict(Nx=n, Ny=n, Nz=n, Nc_fundamental=2, Kn=1.0, pressDrop=1.0, eps=1e-8, chkConvergeStep=10,
             maxStep=1000, wallExtOrder=2)
    d.update(kw)
    return pk.default_params(**d)
