"""Shared fixtures. GPU tests carry ``@pytest.mark.gpu``; everything else runs on the CPU."""
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (os.path.join(ROOT, "oracle"), os.path.join(ROOT, "wsl-code_b200"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(GOLDEN, "golden.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def square_meshes():
    z = np.load(os.path.join(GOLDEN, "square_meshes.npz"))
    names = sorted({k.split("/")[0] for k in z.files})
    return {n: dict(xy=z[n + "/xy"], cell_ptr=z[n + "/cell_ptr"], cell_nodes=z[n + "/cell_nodes"]) for n in names}


@pytest.fixture(scope="session")
def ref_blocks():
    return np.load(os.path.join(GOLDEN, "ref_blocks.npz"))
