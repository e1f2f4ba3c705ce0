"""GPU: pdgpu_md_run_io (MD with the state in host memory) gives the same
bits as the separate calls it replaces: set positions and velocities,
pdgpu_md_run, get positions, velocities and energies."""
import ctypes

import numpy as np
import pytest

from conftest import build_workspace, load_fixture

pytestmark = pytest.mark.gpu


def test_md_run_io_equals_separate_calls(gpu_ctx):
    from pdgpu import _abi as A
    L = A.lib()
    arrays, meta = load_fixture("c1_pep64_s0")
    ws, ff = build_workspace(arrays, meta, gpu_ctx)
    ws.nlist().calcNewList()
    n = ws.nAtoms()
    p = A.md_params_default()
    p.Integrator, p.UpdateNList, p.UseGraph = A.INTEGRATOR_LANGEVIN, 10, 1
    p.Timestep, p.FricCoeff, p.TargetTemp, p.Seed = 1e-15, 1e12, 300.0, 3
    A.check(L.pdgpu_md_init_velocities(gpu_ctx.ptr, ws._sys, 300.0, 3))
    x0, v0 = np.zeros((n, 3)), np.zeros((n, 3))
    A.check(L.pdgpu_get_positions(gpu_ctx.ptr, ws._sys, A.dptr(x0)))
    A.check(L.pdgpu_get_velocities(gpu_ctx.ptr, ws._sys, A.dptr(v0)))
    outs = []
    for fused in (False, True, True):  # two fused calls in a row
        x, v, e = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(A.ENE_COUNT)
        if fused:
            A.check(L.pdgpu_md_run_io(gpu_ctx.ptr, ws._sys, ctypes.byref(p), 0, 20, 20, A.dptr(x0), A.dptr(v0),
                                      A.dptr(x), A.dptr(v), A.dptr(e)))
        else:
            A.check(L.pdgpu_set_positions(gpu_ctx.ptr, ws._sys, A.dptr(x0)))
            A.check(L.pdgpu_set_velocities(gpu_ctx.ptr, ws._sys, A.dptr(v0)))
            A.check(L.pdgpu_md_run(gpu_ctx.ptr, ws._sys, ctypes.byref(p), 0, 20, 20, None))
            A.check(L.pdgpu_get_positions(gpu_ctx.ptr, ws._sys, A.dptr(x)))
            A.check(L.pdgpu_get_velocities(gpu_ctx.ptr, ws._sys, A.dptr(v)))
            A.check(L.pdgpu_get_energies(gpu_ctx.ptr, ws._sys, A.dptr(e), A.ENE_COUNT))
        outs.append((x, v, e))
    assert np.all(np.isfinite(outs[0][0])) and not np.array_equal(outs[0][0], x0)
    for x, v, e in outs[1:]:
        assert np.array_equal(x, outs[0][0])
        assert np.array_equal(v, outs[0][1])
        assert np.array_equal(e, outs[0][2])
    ws.close()
