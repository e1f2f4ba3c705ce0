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


def _md_positions(ctx, arrays, meta, use_graph, cuts):
    """Positions after MD runs of the given lengths back to back (one
    handle), each call starting where the last one stopped."""
    from pdgpu import _abi as A
    L = A.lib()
    ws, ff = build_workspace(arrays, meta, ctx)
    ws.nlist().calcNewList()
    n = ws.nAtoms()
    p = A.md_params_default()
    p.Integrator, p.UpdateNList, p.UseGraph = A.INTEGRATOR_LANGEVIN, 10, use_graph
    p.Timestep, p.FricCoeff, p.TargetTemp, p.Seed = 1e-15, 1e12, 300.0, 5
    A.check(L.pdgpu_md_init_velocities(ctx.ptr, ws._sys, 300.0, 5))
    total = sum(cuts)
    s = 0
    replays = []
    for k in cuts:
        A.check(L.pdgpu_md_run(ctx.ptr, ws._sys, ctypes.byref(p), s, k, total, None))
        s += k
        r = np.zeros(2, dtype=np.int64)
        A.check(L.pdgpu_graph_replays(ctx.ptr, ws._sys, r.ctypes.data_as(A._I64)))
        replays.append(int(r[0]))
    x = np.zeros((n, 3))
    A.check(L.pdgpu_get_positions(ctx.ptr, ws._sys, A.dptr(x)))
    e = np.zeros(A.ENE_COUNT)
    A.check(L.pdgpu_get_energies(ctx.ptr, ws._sys, A.dptr(e), A.ENE_COUNT))
    ws.close()
    return x, e, replays


def test_md_run_mid_period_replays_graphs(gpu_ctx):
    """A run that starts inside a list period (5 warm-up steps, then 10 and
    7) replays graphs for its partial head block, the whole period and the
    partial tail, and gives the same bits as the same steps run eagerly."""
    arrays, meta = load_fixture("c1_pep64_s0")
    cuts = [5, 10, 7]
    xg, eg, rg = _md_positions(gpu_ctx, arrays, meta, 1, cuts)
    xe, ee, re_ = _md_positions(gpu_ctx, arrays, meta, 0, cuts)
    assert np.all(np.isfinite(xg))
    assert np.array_equal(xg, xe) and np.array_equal(eg, ee)
    assert re_ == [0, 0, 0]
    # 5 steps: one block [rebuild + 5]; 10 steps from step 5: [5 without
    # rebuild] + [rebuild + 5]; 7 steps from step 15: [5] + [rebuild + 2]
    assert rg == [1, 3, 5]
