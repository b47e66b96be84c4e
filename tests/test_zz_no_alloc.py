"""The allocation-free sort entry point (cudasph_radix_sort_u64_noalloc).

Some callers cannot allocate device memory themselves (their host framework
owns all of it, or cudaMalloc would stall a time-critical loop), so this entry
point takes only the keys and values and works in a scratch array compiled
into the library.  Its results must be identical -- bit for bit, as for every
integer result here -- to the allocating entry point's, call after call, since
all calls share that array.  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_KEYS = 262144  # CUDASPH_SORT_NOALLOC_MAX_KEYS


def _lib():
    from cudasph_b200._capi import lib
    L = lib()
    L.cudasph_radix_sort_u64_noalloc.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    return L


def _keys(n, seed):
    rs = np.random.default_rng(seed)
    k = rs.integers(0, 1 << 63, size=n, dtype=np.int64)
    q = n // 4
    k[:q] = k[q:2 * q]  # many equal keys: ties must keep input order
    return k


def test_noalloc_sort_matches_allocating_sort_twice():
    """Two calls in a row (different sizes, the second at the maximum) equal
    the allocating sort bit for bit, and the values are the oracle's stable
    order of the keys."""
    import torch
    from oracle import oracle as O
    L = _lib()
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream().cuda_stream
    for call, (n, seed) in enumerate([(100_003, 1), (MAX_KEYS, 2)]):
        keys = _keys(n, seed)
        k = torch.from_numpy(keys).to(dev)
        v = torch.arange(n, dtype=torch.int32, device=dev)
        k_ref, v_ref = k.clone(), v.clone()
        scratch = torch.empty(L.cudasph_sort_scratch_bytes(n), dtype=torch.uint8, device=dev)
        assert L.cudasph_radix_sort_u64(n, k_ref.data_ptr(), v_ref.data_ptr(), scratch.data_ptr(), stream) == 0
        assert L.cudasph_radix_sort_u64_noalloc(n, k.data_ptr(), v.data_ptr(), stream) == 0
        torch.cuda.synchronize()
        assert torch.equal(k, k_ref), f"call {call}: keys differ"
        assert torch.equal(v, v_ref), f"call {call}: values differ"
        kk = k.cpu().numpy().view(np.uint64)
        assert np.all(kk[1:] >= kk[:-1])
        assert np.array_equal(v.cpu().numpy(), O.sort_order(keys.view(np.uint64))), f"call {call}: not stable"


def test_noalloc_sort_allocates_no_device_memory():
    """After a first call (the address lookup), a call at the maximum size
    leaves the device's free memory unchanged: the scratch is the array
    compiled into the library, not an allocation."""
    import torch
    L = _lib()
    dev = torch.device("cuda:0")
    k = torch.from_numpy(_keys(MAX_KEYS, 3)).to(dev)
    v = torch.arange(MAX_KEYS, dtype=torch.int32, device=dev)
    assert L.cudasph_radix_sort_u64_noalloc(MAX_KEYS, k.data_ptr(), v.data_ptr(), None) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(dev)
    for _ in range(3):
        assert L.cudasph_radix_sort_u64_noalloc(MAX_KEYS, k.data_ptr(), v.data_ptr(), None) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(dev)
    assert free1 == free0


def test_noalloc_sort_rejects_more_keys_than_its_scratch():
    import torch
    L = _lib()
    k = torch.zeros(MAX_KEYS + 1, dtype=torch.int64, device="cuda:0")
    v = torch.zeros(MAX_KEYS + 1, dtype=torch.int32, device="cuda:0")
    assert L.cudasph_radix_sort_u64_noalloc(MAX_KEYS + 1, k.data_ptr(), v.data_ptr(), None) == 2  # SPH_ERR_ARG
    assert b"262144" in L.cudasph_last_error()
