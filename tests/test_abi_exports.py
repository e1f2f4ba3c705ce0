"""CPU: the C-ABI library loads and exports every symbol include/*.h
declares; calls that need a device fail cleanly without one."""
import ctypes
import glob
import os
import re

import pytest

from conftest import ROOT

import pdgpu
from pdgpu import _abi as A


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(pdgpu_[a-z0-9_]+)\s*\(", src))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "pdgpu_nlist_build" in names and "pdgpu_gb_forces" in names
    assert len(names) >= 30


def test_library_exports_every_declared_symbol():
    L = A.lib()
    missing = [n for n in declared_symbols() if not hasattr(L, n)]
    assert not missing, missing


def test_python_prototypes_cover_the_header():
    assert set(declared_symbols()) <= set(A.PROTOTYPES)


def test_defaults_mirror_reference_constructors():
    p = A.ff_params_default()
    # FF_GeneralizedBorn_Still (gbff.cpp:17-38) over FF_NonBonded defaults
    assert (p.DielectricSolvent, p.GbsaStillCutoff, p.ExpApproxThreshold) == (80.0, 10.0, -4.0)
    assert (p.P1, p.P2, p.P3, p.P4, p.P5) == (0.073, 0.921, 6.211, 15.236, 1.254)
    assert p.FastMode == 1 and p.EnergySwitch == 1 and p.ForceSwitch == 0 and p.Padding == 0.5
    m = A.md_params_default()
    assert m.Integrator == A.INTEGRATOR_BEEMAN and m.UpdateNList == 10 and m.Timestep == 1e-15
    assert m.FricCoeff == 10e12
    n = A.min_params_default()
    assert n.Algorithm == A.MIN_CONJUGATE_GRADIENTS and n.StepSize == 2e5 and n.UpdateNList == 1
    c = A.mc_params_default()
    # MonteCarlo (montecarlo.h:52-53): ConstantProfile(300), FinalState LastAcc
    assert c.Temperature == 300.0 and c.FinalState == A.MC_LAST_ACC and c.Steps == 0
    assert abs(c.Sigma - 15.0 * 3.14159265358979323846 / 180.0) < 1e-15


def test_null_arguments_are_rejected_without_a_device():
    L = A.lib()
    assert L.pdgpu_ctx_create(0, None) == A.ERR_ARG
    assert "NULL" in A.last_error()
    assert L.pdgpu_gb_forces(None, 1) == A.ERR_ARG


def test_no_device_is_an_error_not_a_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    ctx = A._CTX()
    st = A.lib().pdgpu_ctx_create(0, ctypes.byref(ctx))
    assert st in (A.ERR_NODEVICE, A.ERR_CUDA)
    with pytest.raises(pdgpu.PdgpuError):
        pdgpu.Context(0)
