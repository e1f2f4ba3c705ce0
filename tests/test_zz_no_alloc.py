"""GPU: the allocation-free neighbour-list build.

pdgpu_nlist_build_noalloc exists for callers that cannot call cudaMalloc:
host frameworks that reserve all device memory for their own pool at
start-up and forbid allocation afterwards.  It must give
the same pair set and bond orders as pdgpu_nlist_build -- compared exactly,
as sorted pair sets, the tolerance every list test uses -- on two calls in a
row (its static scratch keeps the previous call's contents).
"""
import ctypes

import numpy as np
import pytest

from conftest import load_fixture

pytestmark = pytest.mark.gpu


def _rows_sorted(ptr, data):
    out = []
    for i in range(len(ptr) - 1):
        row = data[ptr[i]:ptr[i + 1]]
        out.append(row[np.argsort(row & 0xFFFFFF, kind="stable")])
    return out


@pytest.mark.parametrize("name", ["c1_pep64_s0", "pep30_s3_rc16"])
def test_nlist_noalloc_matches_nlist_build(name):
    import torch
    import pdgpu
    from pdgpu import _abi as A

    arrays, meta = load_fixture(name)
    ctx = pdgpu.Context(0)
    ws = pdgpu.WorkSpace(pdgpu.SystemSpec(arrays, meta), ctx)
    ff = pdgpu.Forcefield(ws)
    gb = pdgpu.FF_GeneralizedBorn_Still(ws)
    gb.Cutoff = gb.VdwCutoff = float(meta["cutoff"])
    gb.InnerCutoff = gb.VdwInnerCutoff = float(meta["inner"])
    ff.add(gb)
    ws.nlist().calcNewList()
    ref_ptr, ref_data = ws.nlist().getData(shadow=True)

    n = ws.nAtoms()
    dev = torch.device("cuda", 0)
    pos = torch.tensor(arrays["pos"], dtype=torch.float64, device=dev)
    x, y, z = (pos[:, k].contiguous() for k in range(3))
    band = torch.tensor(arrays["bo_band"], dtype=torch.int8, device=dev)
    mid = int(arrays["bo_mid"][0])
    cap = len(ref_data) + 64
    row_start = torch.empty(n + 1, dtype=torch.int64, device=dev)
    entries = torch.empty(cap, dtype=torch.int32, device=dev)
    cutoff = max(float(meta["cutoff"]), float(meta["vdwcut"])) + 0.5
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call in range(2):
        entries.fill_(-1)
        count = ctypes.c_int64(0)
        st = A.lib().pdgpu_nlist_build_noalloc(
            x.data_ptr(), y.data_ptr(), z.data_ptr(), n, cutoff, mid, band.data_ptr(), None, None,
            row_start.data_ptr(), entries.data_ptr(), cap, ctypes.byref(count), stream)
        assert st == 0, A.last_error()
        torch.cuda.synchronize()
        assert count.value == len(ref_data)
        ptr = row_start.cpu().numpy().astype(np.int32)
        data = entries[: count.value].cpu().numpy()
        assert np.array_equal(ptr, ref_ptr), "call %d: row offsets differ" % call
        got = _rows_sorted(ptr, data)
        for i in range(n):
            assert np.array_equal(got[i], ref_data[ref_ptr[i]:ref_ptr[i + 1]]), "call %d row %d" % (call, i)
    # too small an output buffer is refused, with the size it needs
    count = ctypes.c_int64(0)
    st = A.lib().pdgpu_nlist_build_noalloc(
        x.data_ptr(), y.data_ptr(), z.data_ptr(), n, cutoff, mid, band.data_ptr(), None, None,
        row_start.data_ptr(), entries.data_ptr(), 10, ctypes.byref(count), stream)
    assert st == A.ERR_ARG and count.value == len(ref_data)
    ws.close()


def test_nlist_noalloc_refuses_oversized_systems():
    from pdgpu import _abi as A
    count = ctypes.c_int64(0)
    st = A.lib().pdgpu_nlist_build_noalloc(None, None, None, 70000, 12.5, 1, None, None, None, None, None, 0,
                                           ctypes.byref(count), None)
    assert st == A.ERR_ARG and "65536" in A.last_error()
