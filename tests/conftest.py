"""Shared test setup: the gpu marker, import paths and fixture loading."""
import glob
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, os.path.join(ROOT, "pd.arcus_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libpdgpu.so")


def fixture_names(small_only=True):
    names = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))
    if small_only:
        names = [n for n in names if not n.startswith("c2_")]
    return names


def load_fixture(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    arrays = {k: z[k] for k in z.files}
    meta = json.loads(bytes(arrays.pop("meta_json")).decode())
    return arrays, meta


def rel_rms(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.sqrt(np.sum((a - b) ** 2) / max(np.sum(b ** 2), 1e-300)))


@pytest.fixture(scope="session")
def gpu_ctx():
    import pdgpu
    return pdgpu.Context(0)
