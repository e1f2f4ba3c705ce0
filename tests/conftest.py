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
    names = [n for n in names if not n.startswith("lib")]  # peptide libraries: load_library
    if small_only:
        names = [n for n in names if not n.startswith("c2_")]
    return names


def load_library(name):
    """A peptide library fixture: list of (arrays, meta) per member."""
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    meta = json.loads(bytes(z["meta_json"]).decode())
    out = []
    for k, m in enumerate(meta["members"]):
        pre = "p%02d_" % k
        arrays = {f[len(pre):]: z[f] for f in z.files if f.startswith(pre)}
        out.append((arrays, m))
    return out


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


def build_workspace(arrays, meta, ctx, with_bonded=True):
    """WorkSpace + Forcefield{FF_Bonded, FF_GeneralizedBorn_Still} with the
    cutoffs the fixture was made with, set up on the device."""
    import pdgpu
    spec = pdgpu.SystemSpec(arrays, meta)
    ws = pdgpu.WorkSpace(spec, ctx)
    ff = pdgpu.Forcefield(ws)
    if with_bonded:
        ff.add(pdgpu.FF_Bonded(ws))
    gb = pdgpu.FF_GeneralizedBorn_Still(ws)
    gb.Cutoff = float(meta["cutoff"])
    gb.InnerCutoff = float(meta["inner"])
    gb.VdwCutoff = float(meta["vdwcut"])
    gb.VdwInnerCutoff = float(meta["vdwinner"])
    ff.add(gb)
    ff.ensuresetup()
    return ws, ff
