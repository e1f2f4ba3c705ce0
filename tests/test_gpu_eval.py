"""GPU: the evaluation kernel on the cluster-pair tiles (Born sums, GB + LJ +
Coulomb and the chain rule as phases of one cooperative launch).

Tolerances:
  one launch vs three launches        bit-exact (the same phases)
  Born radii vs the row passes        bit-exact (the same FP32 terms, each
                                      added in 64-bit fixed point)
  forces vs the row passes            relative RMS 1e-6
  forces vs the reference (FP64)      relative RMS 1e-5
  energies vs the reference           relative 1e-5 or 1e-3 kcal/mol
  repeated evaluations                bit-exact
"""
import ctypes

import numpy as np
import pytest

from conftest import build_workspace, fixture_names, load_fixture, load_library, rel_rms

pytestmark = pytest.mark.gpu

J2K = (1.0 / 4184.0) * 6.0221418e23


def _eval(ws, ff):
    ws.nlist().calcNewList()
    ff.calcForces()
    return ws.cur.f.copy(), ws._pull_energies().copy(), ws.born_radii().copy()


@pytest.mark.parametrize("name", fixture_names() + ["c2_16x80_s2"])
def test_one_launch_equals_three_and_reference(name, gpu_ctx):
    arrays, meta = load_fixture(name)
    ws, ff = build_workspace(arrays, meta, gpu_ctx)
    assert ws.setPairPath(0) == 0
    f_r, e_r, b_r = _eval(ws, ff)
    assert ws.setPairPath(1) == 1
    assert ws.setEvalMode(1) == 1
    f1, e1, b1 = _eval(ws, ff)
    f1b, e1b, b1b = _eval(ws, ff)
    assert ws.setEvalMode(0) == 0
    f3, e3, b3 = _eval(ws, ff)
    assert np.array_equal(f1, f1b) and np.array_equal(e1, e1b) and np.array_equal(b1, b1b)
    assert np.array_equal(f1, f3) and np.array_equal(e1, e3) and np.array_equal(b1, b3)
    assert np.array_equal(b1, b_r)
    assert rel_rms(f1, f_r) <= 1e-6
    assert rel_rms(f1, arrays["f_total"]) <= 1e-5
    e_ref = arrays["ene_total"][0]
    assert abs(e1[0] - e_ref) * J2K <= max(1e-5 * abs(e_ref) * J2K, 1e-3)
    ws.close()


def test_profile_eval_counts(gpu_ctx):
    from pdgpu import _abi as A
    arrays, meta = load_fixture("c2_16x80_s2")
    ws, ff = build_workspace(arrays, meta, gpu_ctx)
    ws.setPairPath(1)
    ws.nlist().calcNewList()
    ff.calcForces()
    ms = np.zeros(4)
    cnt = np.zeros(5, dtype=np.int64)
    A.check(A.lib().pdgpu_profile_eval(gpu_ctx.ptr, ws._sys, 3, A.dptr(ms), cnt.ctypes.data_as(A._I64)))
    assert np.all(ms > 0)
    assert 0 < cnt[1] < cnt[0]  # at Rc 16 some tiles hold no pair inside the 10 A Still cutoff
    # tiles redone in the careful form (a pair at a decision edge): few
    assert np.all(cnt[2:] >= 0) and cnt[2] + cnt[3] < cnt[0] // 4 and cnt[4] < cnt[1] // 4, cnt
    # the evaluation after profiling still gives the reference's forces
    f, e, b = _eval(ws, ff)
    assert rel_rms(f, arrays["f_total"]) <= 1e-5
    ws.close()


def test_batch_one_launch_equals_alone(gpu_ctx):
    import pdgpu
    members = [build_workspace(a, m, gpu_ctx) + (a, m) for a, m in load_library("lib16_amber_s3")[:6]]
    alone = []
    for ws, ff, a, m in members:
        one = pdgpu.Batch([ws])
        one.setPairPath(1)
        f, e = one.evaluate()
        alone.append((f, e[0]))
        one.close()
    b = pdgpu.Batch([ws for ws, *_ in members])
    b.setPairPath(1)
    f, e = b.evaluate()
    for s, (ws, ff, a, m) in enumerate(members):
        assert np.array_equal(b.split(f)[s], alone[s][0])
        assert np.array_equal(e[s], alone[s][1])
        assert rel_rms(b.split(f)[s], a["f_total"]) <= 1e-5
    b.close()


def test_batch_three_launches_equal_one(gpu_ctx):
    import pdgpu
    members = [build_workspace(a, m, gpu_ctx) + (a, m) for a, m in load_library("lib16_opls_s4")[:5]]
    b = pdgpu.Batch([ws for ws, *_ in members])
    b.setPairPath(1)
    assert b.setEvalMode(1) == 1
    f1, e1 = b.evaluate()
    assert b.setEvalMode(0) == 0
    f3, e3 = b.evaluate()
    assert np.array_equal(f1, f3) and np.array_equal(e1, e3)
    b.close()


def test_md_one_launch_equals_three(gpu_ctx):
    """Langevin MD on the tile layout: the step loop with the evaluation in
    one launch and in three gives the same trajectory and energy history
    (the records of consecutive steps alternate between two energy
    buffers)."""
    from pdgpu import _abi as A
    import ctypes
    arrays, meta = load_fixture("c1_pep64_s0")
    out = []
    for mode in (1, 0, 2):
        ws, ff = build_workspace(arrays, meta, gpu_ctx)
        ws.setPairPath(1)
        assert ws.setEvalMode(-1) == 2  # the default
        assert ws.setEvalMode(mode) == mode
        ws.nlist().calcNewList()
        p = A.md_params_default()
        p.Integrator, p.UpdateNList, p.UseGraph = A.INTEGRATOR_LANGEVIN, 10, 1
        p.Timestep, p.FricCoeff, p.TargetTemp, p.Seed = 1e-15, 1e12, 300.0, 11
        A.check(A.lib().pdgpu_md_init_velocities(gpu_ctx.ptr, ws._sys, 300.0, 11))
        hist = np.zeros((25, 3))
        A.check(A.lib().pdgpu_md_run(gpu_ctx.ptr, ws._sys, ctypes.byref(p), 0, 25, 25, A.dptr(hist)))
        x = np.zeros((ws.nAtoms(), 3))
        A.check(A.lib().pdgpu_get_positions(gpu_ctx.ptr, ws._sys, A.dptr(x)))
        ep = np.zeros(ws.nAtoms())
        A.check(A.lib().pdgpu_get_atom_epot(gpu_ctx.ptr, ws._sys, A.dptr(ep)))
        out.append((x, hist, ep))
        ws.close()
    assert np.all(np.isfinite(out[0][0]))
    for q in range(3):
        assert np.array_equal(out[0][q], out[1][q])
        assert np.array_equal(out[0][q], out[2][q])


_LEAN_SCRIPT = r"""
import sys, numpy as np
sys.path.insert(0, sys.argv[1]); sys.path.insert(0, sys.argv[2])
import pdgpu
from conftest import build_workspace, load_fixture
ctx = pdgpu.Context(0)
arrays, meta = load_fixture("c1_pep64_s0")
ws, ff = build_workspace(arrays, meta, ctx)
ws.setPairPath(1)
ws.nlist().calcNewList()
ff.calcForces()
np.save(sys.argv[3], ws.cur.f)
"""


def test_lean_build_equals_general(gpu_ctx, tmp_path):
    """The evaluation kernel's lean build (FastMode, one switch for LJ and
    GB/Coulomb) gives the general build's bits: the general build runs in a
    child process (PDGPU_EV_LEAN=0)."""
    import os
    import subprocess
    import sys
    from conftest import ROOT
    arrays, meta = load_fixture("c1_pep64_s0")
    ws, ff = build_workspace(arrays, meta, gpu_ctx)
    ws.setPairPath(1)
    ws.nlist().calcNewList()
    ff.calcForces()
    out = str(tmp_path / "f_general.npy")
    env = dict(os.environ, PDGPU_EV_LEAN="0")
    subprocess.run([sys.executable, "-c", _LEAN_SCRIPT, os.path.join(ROOT, "pd.arcus_b200"),
                    os.path.join(ROOT, "tests"), out], env=env, check=True, timeout=300)
    assert np.array_equal(np.load(out), ws.cur.f)
    ws.close()


def test_measured_pipe_peaks_are_near_nominal(gpu_ctx):
    """pdgpu_measure_pipe_peaks (the roofline's FP32 and MUFU denominators):
    every SM counted, and each pipe between half and 1.15 x its nominal
    rate at the device's maximum clock (128 FMA and 16 MUFU lanes a SM)."""
    import torch
    from pdgpu import _abi as A
    out = np.zeros(3)
    A.check(A.lib().pdgpu_measure_pipe_peaks(gpu_ctx.ptr, A.dptr(out)))
    props = torch.cuda.get_device_properties(0)
    sms = props.multi_processor_count
    assert int(out[2]) == sms
    import pynvml
    pynvml.nvmlInit()
    f_max = pynvml.nvmlDeviceGetMaxClockInfo(pynvml.nvmlDeviceGetHandleByIndex(0), pynvml.NVML_CLOCK_SM) * 1e6
    assert 0.5 * sms * 256 * f_max <= out[0] <= 1.15 * sms * 256 * f_max
    assert 0.5 * sms * 16 * f_max <= out[1] <= 1.15 * sms * 16 * f_max
