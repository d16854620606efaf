"""GPU: the radix-sort entry point that allocates nothing, against the allocating one.

dipl_radix_sort_pairs_noalloc serves callers that may not allocate device memory (an application that owns
the GPU heap, a loop that must not stall on cudaMalloc); its scratch is a fixed array inside the library.
This file is collected last so that a run stopping at the first failure has run every other test first.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from diplodocus_b200 import _lib as L

pytestmark = pytest.mark.gpu

MAX_PAIRS = 1 << 18


def _sort(fn, keys, vals, end_bit, digit_bits=0):
    lib = L.load()
    n = keys.numel()
    ko = torch.empty_like(keys)
    vo = torch.empty(n, dtype=torch.int32, device=keys.device)
    vp = C.c_void_p(vals.data_ptr()) if vals is not None else C.c_void_p(0)
    st = getattr(lib, fn)(C.c_void_p(keys.data_ptr()), vp, C.c_void_p(ko.data_ptr()), C.c_void_p(vo.data_ptr()), n,
                          keys.element_size(), 0, end_bit, digit_bits,
                          C.c_void_p(torch.cuda.current_stream().cuda_stream))
    return st, ko, vo


@pytest.mark.parametrize("key_bytes,end_bit,digit_bits", [(8, 64, 10), (4, 30, 8), (8, 60, 8)])
def test_noalloc_sort_matches_allocating_sort_on_two_calls(key_bytes, end_bit, digit_bits):
    rng = np.random.default_rng(key_bytes * 100 + end_bit)
    for call, n in enumerate((MAX_PAIRS, 100_003)):
        dt = np.int32 if key_bytes == 4 else np.int64
        keys = rng.integers(0, 1 << min(end_bit, 62), size=n, dtype=np.int64).astype(dt)
        keys[: n // 4] = keys[0]  # duplicates: the sorts are stable
        vals = rng.permutation(n).astype(np.int32)
        kt = torch.from_numpy(keys).cuda()
        vt = torch.from_numpy(vals).cuda()
        st_ref, ko_ref, vo_ref = _sort("dipl_radix_sort_pairs", kt, vt, end_bit, digit_bits)
        st, ko, vo = _sort("dipl_radix_sort_pairs_noalloc", kt, vt, end_bit, digit_bits)
        assert st_ref == L.DIPL_OK and st == L.DIPL_OK, (call, st_ref, st)
        torch.cuda.synchronize()
        # integer work: bit-exact equality is the tolerance
        assert torch.equal(ko, ko_ref), f"keys differ on call {call}"
        assert torch.equal(vo, vo_ref), f"values differ on call {call}"


def test_noalloc_sort_rejects_sizes_beyond_its_limit():
    kt = torch.zeros(MAX_PAIRS + 1, dtype=torch.int32, device="cuda")
    st, _, _ = _sort("dipl_radix_sort_pairs_noalloc", kt, None, 32)
    assert st == 1  # DIPL_ERR_INVALID_ARGUMENT
    assert b"exceeds the limit" in L.load().dipl_last_error()
