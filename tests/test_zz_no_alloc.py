"""GPU: the radix-sort entry point that allocates nothing, against the allocating one.

dipl_radix_sort_pairs_noalloc serves callers that may not allocate device memory (an application that owns
the GPU heap, a loop that must not stall on cudaMalloc); its scratch is a fixed array inside the library.
This file is collected last so that a run stopping at the first failure has run every other test first.
"""
import ctypes as C
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest
import torch

from conftest import ROOT
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


@pytest.mark.parametrize("key_bytes,end_bit", [(4, 32), (8, 60)])
def test_noalloc_sort_without_values_and_empty_input(key_bytes, end_bit):
    """d_vals_in = NULL (values default to 0..n-1, no value array is read) gives the allocating sort's keys and
    values bit for bit, on two calls in a row; n = 0 returns at once."""
    rng = np.random.default_rng(end_bit)
    dt = np.int32 if key_bytes == 4 else np.int64
    for call, n in enumerate((MAX_PAIRS, 77_777)):
        keys = rng.integers(0, 1 << min(end_bit, 31), size=n, dtype=np.int64).astype(dt)
        kt = torch.from_numpy(keys).cuda()
        st_ref, ko_ref, vo_ref = _sort("dipl_radix_sort_pairs", kt, None, end_bit)
        st, ko, vo = _sort("dipl_radix_sort_pairs_noalloc", kt, None, end_bit)
        assert st_ref == L.DIPL_OK and st == L.DIPL_OK, (call, st_ref, st)
        torch.cuda.synchronize()
        assert torch.equal(ko, ko_ref) and torch.equal(vo, vo_ref), f"call {call}"
    empty = torch.empty(0, dtype=torch.int32, device="cuda")
    st, _, _ = _sort("dipl_radix_sort_pairs_noalloc", empty, None, 32)
    assert st == L.DIPL_OK


def test_noalloc_sort_leaves_device_free_memory_unchanged():
    """After the first call has loaded the library's device image, further calls change the device's free memory
    by nothing: the scratch is the fixed array, not an allocation."""
    n = MAX_PAIRS
    keys = torch.from_numpy(np.random.default_rng(3).integers(0, 1 << 40, size=n, dtype=np.int64)).cuda()
    _sort("dipl_radix_sort_pairs_noalloc", keys, None, 64)  # first call: image loaded, address looked up
    lib = L.load()
    ko = torch.empty_like(keys)
    vo = torch.empty(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(5):
        st = lib.dipl_radix_sort_pairs_noalloc(C.c_void_p(keys.data_ptr()), C.c_void_p(0), C.c_void_p(ko.data_ptr()),
                                               C.c_void_p(vo.data_ptr()), n, 8, 0, 64, 0,
                                               C.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert st == L.DIPL_OK
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


_CONTEXT_CHILD = textwrap.dedent("""
    import ctypes as C, sys
    import numpy as np
    sys.path.insert(0, sys.argv[1])
    from cuda.bindings import driver as drv
    from diplodocus_b200 import _lib as L

    def ok(r):
        err = r[0] if isinstance(r, tuple) else r
        assert err == drv.CUresult.CUDA_SUCCESS, err
        return r[1] if isinstance(r, tuple) and len(r) == 2 else r

    lib = L.load()
    ok(drv.cuInit(0))
    dev = ok(drv.cuDeviceGet(0))

    def sort_in_current_context(seed):
        n = 50_000
        keys = np.random.default_rng(seed).integers(0, 1 << 32, size=n, dtype=np.uint64).astype(np.uint32)
        bufs = [ok(drv.cuMemAlloc(n * 4)) for _ in range(3)]
        ok(drv.cuMemcpyHtoD(bufs[0], keys.ctypes.data, n * 4))
        ok(drv.cuCtxSynchronize())
        st = lib.dipl_radix_sort_pairs_noalloc(C.c_void_p(int(bufs[0])), None, C.c_void_p(int(bufs[1])),
                                               C.c_void_p(int(bufs[2])), n, 4, 0, 32, 0, None)
        assert st == 0, lib.dipl_last_error()
        ok(drv.cuCtxSynchronize())
        ko = np.empty(n, np.uint32)
        vo = np.empty(n, np.uint32)
        ok(drv.cuMemcpyDtoH(ko.ctypes.data, bufs[1], n * 4))
        ok(drv.cuMemcpyDtoH(vo.ctypes.data, bufs[2], n * 4))
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(ko, keys[order]) and np.array_equal(vo, order.astype(np.uint32)), seed
        for b in bufs:
            ok(drv.cuMemFree(b))

    primary = ok(drv.cuDevicePrimaryCtxRetain(dev))
    ok(drv.cuCtxSetCurrent(primary))
    sort_in_current_context(1)
    other = ok(drv.cuCtxCreate(0, dev))   # another context on the same device, now current
    sort_in_current_context(2)            # the scratch address is looked up again in this context
    sort_in_current_context(3)
    ok(drv.cuCtxDestroy(other))
    ok(drv.cuCtxSetCurrent(primary))
    sort_in_current_context(4)            # and again back in the primary context
    ok(drv.cuDevicePrimaryCtxRelease(dev))
    print("contexts ok")
""")


def test_noalloc_sort_follows_the_current_context():
    """Each CUDA context loads the library's device image anew, so the fixed array has one address per context.
    In a fresh process the sort runs in the primary context, in a second context created on the same device and
    back in the primary one, each time equal to a stable sort of the keys: the address is looked up again for a
    context the library has not seen. (The driver API is used directly; no torch in the child.)"""
    r = subprocess.run([sys.executable, "-c", _CONTEXT_CHILD, ROOT], capture_output=True, text=True, timeout=300,
                       env=dict(os.environ, CUDA_VISIBLE_DEVICES=os.environ.get("CUDA_VISIBLE_DEVICES", "0")))
    assert r.returncode == 0 and "contexts ok" in r.stdout, r.stdout + r.stderr
