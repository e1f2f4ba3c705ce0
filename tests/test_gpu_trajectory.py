"""GPU: trajectory snapshots (ProtocolBase::UpdateTra, md.cpp:260).

A frame of step s holds the positions after step s; the same protocol run
stopped after step s (steps 0..s of the same total) must give the same
positions, bit for bit (the frames are written by the integrator inside the
step graph and copied out on the pack's second stream).  A host ring too
small for the run keeps the newest frames and reports the rest dropped.
"""
import ctypes

import numpy as np
import pytest

from conftest import build_workspace, load_fixture

pytestmark = pytest.mark.gpu

TOTAL = 30
EVERY = 5


def _params(A):
    p = A.md_params_default()
    p.Integrator, p.UpdateNList, p.UseGraph = A.INTEGRATOR_LANGEVIN, 10, 1
    p.Timestep, p.FricCoeff, p.TargetTemp, p.Seed = 1e-15, 1e12, 300.0, 11
    return p


def _fresh(gpu_ctx, path):
    arrays, meta = load_fixture("c1_pep64_s0")
    ws, ff = build_workspace(arrays, meta, gpu_ctx)
    ws.setPairPath(path)
    ws.nlist().calcNewList()
    from pdgpu import _abi as A
    A.check(A.lib().pdgpu_md_init_velocities(gpu_ctx.ptr, ws._sys, 300.0, 11))
    return ws


def _positions(ws):
    from pdgpu import _abi as A
    x = np.zeros((ws.nAtoms(), 3))
    A.check(A.lib().pdgpu_get_positions(ws.ctx.ptr, ws._sys, A.dptr(x)))
    return x


@pytest.mark.parametrize("path", [1, 0])
def test_frames_are_the_positions_after_their_steps(gpu_ctx, path):
    from pdgpu import _abi as A
    from pdgpu.core import read_trajectory
    L = A.lib()
    ws = _fresh(gpu_ctx, path)
    A.check(L.pdgpu_md_set_trajectory(gpu_ctx.ptr, ws._sys, EVERY, 16))
    A.check(L.pdgpu_md_run(gpu_ctx.ptr, ws._sys, ctypes.byref(_params(A)), 0, TOTAL, TOTAL, None))
    (frames, steps), dropped = read_trajectory(gpu_ctx, ws._sys, ws.nAtoms(), 16)
    assert dropped == 0
    assert list(steps) == list(range(EVERY, TOTAL, EVERY))  # s > 0, s % every == 0
    for s in (5, 20):
        one = _fresh(gpu_ctx, path)
        A.check(L.pdgpu_md_run(gpu_ctx.ptr, one._sys, ctypes.byref(_params(A)), 0, s + 1, TOTAL, None))
        k = list(steps).index(s)
        assert np.array_equal(frames[k], _positions(one)), s
        one.close()
    # nothing new since the last read
    (frames2, _), dropped2 = read_trajectory(gpu_ctx, ws._sys, ws.nAtoms(), 16)
    assert len(frames2) == 0 and dropped2 == 0
    A.check(L.pdgpu_md_set_trajectory(gpu_ctx.ptr, ws._sys, 0, 0))
    ws.close()


def test_small_ring_keeps_the_newest_frames(gpu_ctx):
    from pdgpu import _abi as A
    from pdgpu.core import read_trajectory
    L = A.lib()
    ws = _fresh(gpu_ctx, 1)
    A.check(L.pdgpu_md_set_trajectory(gpu_ctx.ptr, ws._sys, 1, 4))  # every step, 4 frames kept
    A.check(L.pdgpu_md_run(gpu_ctx.ptr, ws._sys, ctypes.byref(_params(A)), 0, TOTAL, TOTAL, None))
    (frames, steps), dropped = read_trajectory(gpu_ctx, ws._sys, ws.nAtoms(), 8)
    assert list(steps) == [TOTAL - 4, TOTAL - 3, TOTAL - 2, TOTAL - 1]
    assert dropped == (TOTAL - 1) - 4
    assert np.array_equal(frames[-1], _positions(ws))
    ws.close()


def test_protocol_surface(gpu_ctx):
    import pdgpu
    arrays, meta = load_fixture("c1_pep64_s0")
    ws, ff = build_workspace(arrays, meta, gpu_ctx)
    md = pdgpu.MolecularDynamics(ff)
    md.Integrator = pdgpu.MolecularDynamics.Langevin
    md.FricCoeff = 1e12
    md.Steps = 20
    md.UpdateTra = 4
    md.run()
    frames, steps = md.frames
    assert list(steps) == [4, 8, 12, 16]
    assert frames.shape == (4, ws.nAtoms(), 3) and np.all(np.isfinite(frames))
