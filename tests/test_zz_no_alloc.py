"""GPU: the allocation-free neighbour-list build.

pdgpu_nlist_build_noalloc exists for callers that cannot call cudaMalloc:
host frameworks that reserve all device memory for their own pool at
start-up and forbid allocation afterwards.  It must give
the same pair set and bond orders as pdgpu_nlist_build -- compared exactly,
as sorted pair sets, the tolerance every list test uses -- on two calls in a
row (its static scratch keeps the previous call's contents), and the second
call must leave the device's free memory and the default pool's usage (and
its high-water mark) where they were.
"""
import ctypes

import numpy as np
import pytest

from conftest import load_fixture

pytestmark = pytest.mark.gpu


def _pool_usage():
    """(used, high-water) bytes of device 0's default memory pool, through
    the driver API (the pool stream-ordered allocations come from)."""
    cu = ctypes.CDLL("libcuda.so.1")
    dev = ctypes.c_int(0)
    assert cu.cuDeviceGet(ctypes.byref(dev), 0) == 0
    pool = ctypes.c_void_p()
    assert cu.cuDeviceGetDefaultMemPool(ctypes.byref(pool), dev) == 0
    used, high = ctypes.c_uint64(0), ctypes.c_uint64(0)
    assert cu.cuMemPoolGetAttribute(pool, 7, ctypes.byref(used)) == 0   # CU_MEMPOOL_ATTR_USED_MEM_CURRENT
    assert cu.cuMemPoolGetAttribute(pool, 8, ctypes.byref(high)) == 0   # CU_MEMPOOL_ATTR_USED_MEM_HIGH
    return used.value, high.value


def _reset_pool_high():
    cu = ctypes.CDLL("libcuda.so.1")
    dev = ctypes.c_int(0)
    assert cu.cuDeviceGet(ctypes.byref(dev), 0) == 0
    pool = ctypes.c_void_p()
    assert cu.cuDeviceGetDefaultMemPool(ctypes.byref(pool), dev) == 0
    zero = ctypes.c_uint64(0)  # setting the high-water mark to 0 resets it to the current use
    assert cu.cuMemPoolSetAttribute(pool, 8, ctypes.byref(zero)) == 0


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
        torch.cuda.synchronize()
        if call == 1:  # the first call has run: no further call takes device memory
            free0 = torch.cuda.mem_get_info(0)[0]
            _reset_pool_high()
            used0, _ = _pool_usage()
        count = ctypes.c_int64(0)
        st = A.lib().pdgpu_nlist_build_noalloc(
            x.data_ptr(), y.data_ptr(), z.data_ptr(), n, cutoff, mid, band.data_ptr(), None, None,
            row_start.data_ptr(), entries.data_ptr(), cap, ctypes.byref(count), stream)
        assert st == 0, A.last_error()
        torch.cuda.synchronize()
        if call == 1:
            used1, high1 = _pool_usage()
            assert torch.cuda.mem_get_info(0)[0] == free0, "the call changed the device's free memory"
            assert used1 == used0 and high1 == used0, "the call allocated from the default pool"
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
