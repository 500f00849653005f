"""The allocation-free sort entry point, for callers that cannot allocate device memory (cudaMalloc forbidden or too
costly where they run): it must return what the regular entry point returns, call after call, although every call
reuses the same built-in scratch array. Collected last so that a failure here comes after every other test."""
import ctypes as C

import numpy as np
import pytest

from bevy_xpbd_b200 import _native as N

pytestmark = pytest.mark.gpu


def _vp(t):
    return C.c_void_p(t.data_ptr())


def _sort_regular(L, torch, kin, vin, passes):
    n = kin.numel()
    kout, vout = torch.empty_like(kin), torch.empty_like(vin)
    nbytes = L.xpbd_radix_sort_scratch_bytes(n)
    scratch = torch.empty(max(nbytes, 1), dtype=torch.uint8, device="cuda")
    st = L.xpbd_radix_sort_pairs(_vp(kin), _vp(vin), _vp(kout), _vp(vout), n, passes, _vp(scratch), nbytes,
                                 C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0
    return kout, vout


def _sort_noalloc(L, torch, kin, vin, passes):
    kout, vout = torch.empty_like(kin), torch.empty_like(vin)
    st = L.xpbd_radix_sort_pairs_noalloc(_vp(kin), _vp(vin), _vp(kout), _vp(vout), kin.numel(), passes,
                                         C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0
    return kout, vout


def test_noalloc_sort_matches_regular_sort_on_consecutive_calls():
    import torch
    L = N.load()
    rng = np.random.default_rng(11)
    # two calls in a row with different data; the second must not be disturbed by what the first left behind
    for n, hi, passes in [(N.NOALLOC_SORT_MAX_KEYS, 1 << 20, 4), (70_001, 1 << 32, 4), (1, 9, 1)]:
        keys = rng.integers(0, hi, n, dtype=np.uint64).astype(np.uint32)
        kin = torch.from_numpy(keys.view(np.int32)).cuda()
        vin = torch.from_numpy(rng.permutation(n).astype(np.int32)).cuda()
        ka, va = _sort_regular(L, torch, kin, vin, passes)
        kb, vb = _sort_noalloc(L, torch, kin, vin, passes)
        torch.cuda.synchronize()
        assert torch.equal(ka, kb) and torch.equal(va, vb)
        if passes == 4:
            order = np.argsort(keys, kind="stable")
            assert np.array_equal(kb.cpu().numpy().view(np.uint32), keys[order])


def test_noalloc_sort_rejects_more_keys_than_its_scratch_holds():
    import torch
    L = N.load()
    n = N.NOALLOC_SORT_MAX_KEYS + 1
    bufs = [torch.zeros(n, dtype=torch.int32, device="cuda") for _ in range(4)]  # distinct, kept alive
    st = L.xpbd_radix_sort_pairs_noalloc(*[_vp(b) for b in bufs], n, 4, None)
    assert st == N.ERR_CAPACITY
