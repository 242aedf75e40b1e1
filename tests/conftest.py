"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on CPU."""
import importlib
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libfvm2d.so")


@pytest.fixture(scope="session")
def pkg():
    """The product package; builds libfvm2d.so in-tree if it is missing."""
    lib = os.path.join(ROOT, "2d_fvm_cuda_b200", "lib", "libfvm2d.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "2d_fvm_cuda_b200")], check=True)
    return importlib.import_module("2d_fvm_cuda_b200")


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def golden():
    import json
    import numpy as np
    z = np.load(os.path.join(ROOT, "tests", "golden", "reference_cases.npz"))
    manifest = json.loads(bytes(z["manifest"]).decode())
    return z, manifest
