"""The allocation-free sort entry point (luc_sort_u32_static).

For callers that cannot call cudaMalloc — a host that reserves all device
memory when it starts, or a frame loop where an allocation would stall the
device — the library offers one sort whose scratch is a static device array.
These tests call it through the C ABI on caller-owned device arrays and check
its output against the allocating entry point (luc_sort_u32) on two calls in
a row: the scratch is shared and keeps the previous call's contents, so the
second call proves the per-call clearing. Sorting is exact, so the
comparison is exact. This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from lucida_b200 import native


def _err():
    return C.create_string_buffer(256)


def test_rejects_sizes_beyond_the_static_maximum():
    L = native.lib()
    mx = L.luc_sort_u32_static_max()
    assert mx == 1 << 20
    buf = _err()
    rc = L.luc_sort_u32_static(None, None, mx + 1, None, buf, 256)
    assert rc == -4  # LUC_ERR_VALIDATION
    assert b"exceeds the static scratch maximum" in buf.value


@pytest.mark.gpu
def test_static_sort_matches_allocating_sort_twice():
    import torch
    import lucida_b200 as lb

    gpu = lb.Gpu(0)
    L = native.lib()
    stream = torch.cuda.current_stream()
    for call, (n, hi, seed) in enumerate([(300_001, 2**32, 11), ((1 << 20), 1 << 12, 12)]):
        rng = np.random.default_rng(seed)
        keys = rng.integers(0, hi, n, dtype=np.uint64).astype(np.uint32)
        vals = rng.permutation(n).astype(np.uint32)
        ref_k, ref_v = lb.LbvhBuilder(gpu).sort(keys, vals)  # the existing entry point
        dk = torch.from_numpy(keys.view(np.int32)).cuda()
        dv = torch.from_numpy(vals.view(np.int32)).cuda()
        torch.cuda.synchronize()
        buf = _err()
        rc = L.luc_sort_u32_static(C.c_void_p(dk.data_ptr()), C.c_void_p(dv.data_ptr()), n,
                                   C.c_void_p(stream.cuda_stream), buf, 256)
        assert rc == 0, (call, rc, buf.value)
        got_k = dk.cpu().numpy().view(np.uint32)
        got_v = dv.cpu().numpy().view(np.uint32)
        np.testing.assert_array_equal(got_k, ref_k, err_msg=f"keys, call {call}")
        np.testing.assert_array_equal(got_v, ref_v, err_msg=f"values, call {call}")
    gpu.close()
