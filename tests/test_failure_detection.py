"""Failure detection without a GPU fault: every device-side wait of the library is bounded.

The self-test entry point runs the real wait primitives (warp and block decoupled look-back, grid barrier) on a
status word nothing publishes and on a barrier with a participant that never arrives; each must give up after
its poll limit, report DIPL_ERR_TIMEOUT to the host and leave the CUDA context usable for the next build and
trace. No kernel traps, asserts or touches a bad address.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from diplodocus_b200 import _lib as L

DIPL_ERR_INVALID_ARGUMENT, DIPL_ERR_TIMEOUT = 1, 4


def test_selftest_checks_arguments_before_any_gpu_work():
    lib = L.load()
    flags = C.c_uint32(99)
    assert lib.dipl_selftest_bounded_waits(0, C.byref(flags), None) == DIPL_ERR_INVALID_ARGUMENT
    assert lib.dipl_selftest_bounded_waits((1 << 20) + 1, C.byref(flags), None) == DIPL_ERR_INVALID_ARGUMENT
    assert lib.dipl_selftest_bounded_waits(100, None, None) == DIPL_ERR_INVALID_ARGUMENT
    assert b"spin_limit" in lib.dipl_last_error() or b"out_flags" in lib.dipl_last_error()


@pytest.mark.gpu
@pytest.mark.parametrize("spin_limit", [1, 1000])
def test_every_bounded_wait_gives_up_and_the_context_survives(orc, spin_limit):
    lib = L.load()
    torch.cuda.init()
    stream = torch.cuda.current_stream().cuda_stream
    flags = C.c_uint32(0)
    st = lib.dipl_selftest_bounded_waits(spin_limit, C.byref(flags), C.c_void_p(stream))
    assert flags.value == 0b1111, (flags.value, lib.dipl_last_error())
    assert st == DIPL_ERR_TIMEOUT
    # the context still builds and traces correctly after the timeouts
    from gpu_util import build, trace
    from diplodocus_b200 import scenes as S
    tris = S.open_box()
    rays = S.random_rays(256, seed=3)
    h = orc.brute(tris, rays)
    prim, t, _, _ = trace(build(tris), rays)
    np.testing.assert_array_equal(prim, h.prim)
