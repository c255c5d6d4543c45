"""The allocation-free key sort (sphb_sort_by_key_static), for callers that cannot allocate device memory: code
whose device memory all belongs to another allocator, or code running where cudaMalloc is not allowed.

It must give exactly the result of the regular sphb_sort_by_key (which takes caller scratch), on two calls in a row
(the shared scratch array keeps the previous call's contents), leave the device's free memory unchanged, and refuse
sizes beyond its fixed capacity. This file is named so that pytest collects it last; it also passes on its own in a
fresh process.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sort_regular(lib, L, torch, keys):
    n = keys.size
    dk = torch.from_numpy(keys.view(np.int64).copy()).cuda()
    dv = torch.zeros(n, dtype=torch.int32, device="cuda")
    nbytes = lib.sphb_sort_by_key_scratch_bytes(n)
    scratch = torch.empty(max(nbytes, 1), dtype=torch.uint8, device="cuda")
    L.check(lib.sphb_sort_by_key(L.ptr(dk), L.ptr(dv), n, 1, L.ptr(scratch), nbytes, None), "sort")
    torch.cuda.synchronize()
    return dk.cpu().numpy().view(np.uint64), dv.cpu().numpy().view(np.uint32)


def _sort_static(lib, L, torch, keys):
    n = keys.size
    dk = torch.from_numpy(keys.view(np.int64).copy()).cuda()
    dv = torch.zeros(n, dtype=torch.int32, device="cuda")
    L.check(lib.sphb_sort_by_key_static(L.ptr(dk), L.ptr(dv), n, 1, None), "sort_static")
    torch.cuda.synchronize()
    return dk.cpu().numpy().view(np.uint64), dv.cpu().numpy().view(np.uint32)


def test_static_sort_matches_regular_sort_twice(cuda_device):
    import torch
    from sphexa_b200 import lib as L
    lib = L.load()
    cap = lib.sphb_sort_by_key_static_max()
    rng = np.random.default_rng(11)
    # first call: the full capacity with many equal keys (stability) and a removal key
    k1 = rng.integers(0, 2 ** 63, cap, dtype=np.uint64)
    k1[::5] = k1[1]
    k1[7] = np.uint64(1 << 63)
    # second call: a smaller, differently distributed input, so stale scratch from the first call would show
    k2 = (rng.integers(0, 2 ** 20, 300_001, dtype=np.uint64) << np.uint64(40))
    for keys in (k1, k2):
        ks, vs = _sort_static(lib, L, torch, keys)
        kr, vr = _sort_regular(lib, L, torch, keys)
        assert np.array_equal(ks, kr)
        assert np.array_equal(vs, vr)
        perm = np.argsort(keys, kind="stable")
        assert np.array_equal(vs, perm.astype(np.uint32))


def test_static_sort_rejects_oversize(cuda_device):
    import torch
    from sphexa_b200 import lib as L
    lib = L.load()
    cap = lib.sphb_sort_by_key_static_max()
    dk = torch.zeros(cap + 1, dtype=torch.int64, device="cuda")
    dv = torch.zeros(cap + 1, dtype=torch.int32, device="cuda")
    rc = lib.sphb_sort_by_key_static(L.ptr(dk), L.ptr(dv), cap + 1, 1, None)
    assert rc == L.SPHB_ERR_CAPACITY


def test_static_sort_allocates_nothing(cuda_device):
    """After a first call (which looks up the array's address), further calls leave the device's free memory
    exactly as it was: nothing is allocated, not even transiently kept."""
    import torch
    from sphexa_b200 import lib as L
    lib = L.load()
    n = 200_003
    keys = np.random.default_rng(5).integers(0, 2 ** 62, n, dtype=np.uint64)
    dk = torch.from_numpy(keys.view(np.int64).copy()).cuda()
    dv = torch.zeros(n, dtype=torch.int32, device="cuda")
    L.check(lib.sphb_sort_by_key_static(L.ptr(dk), L.ptr(dv), n, 1, None), "sort_static")
    torch.cuda.synchronize()
    host_keys = torch.from_numpy(keys.view(np.int64).copy())
    perm = np.argsort(keys, kind="stable").astype(np.uint32)
    for _ in range(3):
        dk.copy_(host_keys)
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        L.check(lib.sphb_sort_by_key_static(L.ptr(dk), L.ptr(dv), n, 1, None), "sort_static")
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        assert free1 == free0
        assert np.array_equal(dv.cpu().numpy().view(np.uint32), perm)
