"""The allocation-free sort entry point.

mhpc_sort_pairs_noalloc serves callers that cannot allocate device memory
(their own pool reserved the GPU, or allocation is forbidden after start-up):
its scratch is a fixed device array inside the library.  This test calls it
through the C ABI twice in a row (the array keeps the previous call's
contents, so the second call checks that the entry point clears what must
start at zero) and compares each result with the allocating entry point
mhpc_sort_pairs, bit for bit like every sort test here.  It lives in a file
that pytest collects last and passes both alone in a fresh process and after
the other tests.
"""
import ctypes

import numpy as np
import pytest
import torch

from miluphpc_b200 import _lib

pytestmark = pytest.mark.gpu


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _sort_alloc(kin, vin):
    L = _lib.load()
    n = kin.numel()
    kout = torch.empty_like(kin)
    vout = torch.empty(n, dtype=torch.int32, device=kin.device)
    nb = L.mhpc_sort_scratch_bytes(n)
    scratch = torch.empty(nb, dtype=torch.uint8, device=kin.device)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.check(L.mhpc_sort_pairs(_p(kin), _p(vin), _p(kout), _p(vout), n, _p(scratch), nb, s), "sort_pairs")
    return kout, vout


def _sort_noalloc(kin, vin):
    L = _lib.load()
    n = kin.numel()
    kout = torch.empty_like(kin)
    vout = torch.empty(n, dtype=torch.int32, device=kin.device)
    status = torch.full((1,), -1, dtype=torch.int32, device=kin.device)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.check(L.mhpc_sort_pairs_noalloc(_p(kin), _p(vin), _p(kout), _p(vout), n, _p(status), s),
               "sort_pairs_noalloc")
    return kout, vout, status


def test_noalloc_sort_matches_allocating_sort(cuda):
    L = _lib.load()
    nmax = L.mhpc_sort_noalloc_max_n()
    assert nmax == 1 << 20
    rng = np.random.default_rng(42)
    # two calls in a row: a large one, then a smaller one with many equal keys
    cases = [
        (rng.integers(0, 2 ** 63 - 1, size=nmax, dtype=np.int64), None),
        (rng.integers(0, 1000, size=300_001, dtype=np.int64) << 20,
         rng.permutation(300_001).astype(np.int32)),
    ]
    for keys, vals in cases:
        kin = torch.as_tensor(keys, device=cuda)
        vin = torch.as_tensor(vals, device=cuda) if vals is not None else None
        ka, va = _sort_alloc(kin, vin)
        kb, vb, status = _sort_noalloc(kin, vin)
        torch.cuda.synchronize()
        assert int(status.item()) == 0
        assert torch.equal(ka, kb)
        assert torch.equal(va, vb)
        # and both agree with a stable CPU sort
        order = np.argsort(keys.view(np.uint64), kind="stable")
        assert np.array_equal(kb.cpu().numpy(), keys[order])


def test_noalloc_sort_rejects_oversize(cuda):
    L = _lib.load()
    n = L.mhpc_sort_noalloc_max_n() + 1
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = L.mhpc_sort_pairs_noalloc(None, None, None, None, n, None, s)
    assert rc == 3  # MHPC_ERR_CAPACITY, before touching any pointer
    assert L.mhpc_sort_pairs_noalloc(None, None, None, None, 0, None, s) == 0
