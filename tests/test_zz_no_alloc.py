"""GPU test of mpm_radix_sort_u32_noalloc, the sort for callers that cannot allocate.

Callers running under a memory budget fixed up front, or unable to absorb
cudaMalloc/cudaFree latency, use this entry point: it sorts device arrays with a
scratch area compiled into the library.  Its output must equal a CPU stable sort
(numpy.argsort, kind="stable") and that of mpm_radix_sort_u32 (the allocating
entry point) exactly, and it must keep doing so on the next call, which reuses
the same scratch.  Sorting is integer work, so the comparison is bit-exact.
This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_KEYS = 262144   # MPM_NOALLOC_MAX_KEYS in include/mpm_capi.h


def noalloc_sort(L, keys_np, bits):
    import torch
    n = keys_np.size
    dk = torch.from_numpy(keys_np.view(np.int32).copy()).cuda()
    ds = torch.empty(n, dtype=torch.int32, device="cuda")
    dp = torch.empty(n, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    rc = L.mpm_radix_sort_u32_noalloc(ctypes.c_void_p(dk.data_ptr()), ctypes.c_int64(n), bits,
                                      ctypes.c_void_p(ds.data_ptr()), ctypes.c_void_p(dp.data_ptr()),
                                      ctypes.c_void_p(stream.cuda_stream))
    assert rc == 0, rc
    return ds.cpu().numpy().view(np.uint32), dp.cpu().numpy().view(np.uint32)


def test_noalloc_sort_matches_allocating_sort_twice(cuda_device):
    from physbam_b200 import driver as D
    L = D.load_library()
    L.mpm_radix_sort_u32_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_void_p,
                                             ctypes.c_void_p, ctypes.c_void_p]
    L.mpm_radix_sort_u32_noalloc.restype = ctypes.c_int
    rng = np.random.default_rng(2024)
    cases = [(MAX_KEYS, 22), (100_003, 25)]          # two calls in a row on the shared scratch
    for n, bits in cases:
        keys = rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32)
        keys[::5] = keys[7]                          # duplicates: stability matters
        got_k, got_p = noalloc_sort(L, keys, bits)
        low = keys & np.uint32((1 << bits) - 1 if bits < 32 else 0xffffffff)
        cpu_p = np.argsort(low, kind="stable").astype(np.uint32)
        np.testing.assert_array_equal(got_p, cpu_p)
        np.testing.assert_array_equal(got_k, keys[cpu_p])
        ref_k, ref_p = D.radix_sort_u32(keys, bits)
        np.testing.assert_array_equal(got_p, ref_p)
        np.testing.assert_array_equal(got_k, ref_k)


def test_noalloc_sort_rejects_aliased_outputs(cuda_device):
    import torch
    from physbam_b200 import driver as D
    L = D.load_library()
    L.mpm_radix_sort_u32_noalloc.restype = ctypes.c_int
    d = torch.zeros(1000, dtype=torch.int32, device="cuda")
    o = torch.zeros(1000, dtype=torch.int32, device="cuda")
    rc = L.mpm_radix_sort_u32_noalloc(ctypes.c_void_p(d.data_ptr()), ctypes.c_int64(1000), 16,
                                      ctypes.c_void_p(o.data_ptr()), ctypes.c_void_p(o.data_ptr()), None)
    assert rc == 1


def test_noalloc_sort_rejects_too_many_keys(cuda_device):
    import torch
    from physbam_b200 import driver as D
    L = D.load_library()
    L.mpm_radix_sort_u32_noalloc.restype = ctypes.c_int
    n = MAX_KEYS + 1
    d = torch.zeros(n, dtype=torch.int32, device="cuda")
    o = torch.zeros(n, dtype=torch.int32, device="cuda")
    p = torch.zeros(n, dtype=torch.int32, device="cuda")
    rc = L.mpm_radix_sort_u32_noalloc(ctypes.c_void_p(d.data_ptr()), ctypes.c_int64(n), 16,
                                      ctypes.c_void_p(o.data_ptr()), ctypes.c_void_p(p.data_ptr()), None)
    assert rc == 1
