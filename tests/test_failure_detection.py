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


# ---- host-set limits: out of memory, clustering that does not converge, rays that take too many steps --------
# Each failure is made by a limit the host sets (dipl_set_limits), never by a fault: the library reports the status
# a real failure would give, releases what it took, and the context goes on building and tracing correctly.

DIPL_ERR_OUT_OF_MEMORY, DIPL_ERR_INTERNAL = 3, 5


@pytest.fixture
def limits():
    L.set_limits()
    yield L.set_limits
    L.set_limits()


def test_limits_round_trip_on_the_host(limits):
    """The limits are process-wide host state: set, read back, cleared, with no device involved."""
    limits(device_memory_bytes=123456789, clustering_iterations=7, trace_steps=99)
    lim, _ = L.get_limits()
    assert (lim.device_memory_bytes, lim.clustering_iterations, lim.trace_steps) == (123456789, 7, 99)
    limits()
    lim, _ = L.get_limits()
    assert (lim.device_memory_bytes, lim.clustering_iterations, lim.trace_steps) == (0, 0, 0)
    assert L.load().dipl_set_limits(None) == DIPL_ERR_INVALID_ARGUMENT


def _check_build_and_trace(orc, tris, rays, **kw):
    from gpu_util import build, fbits, trace
    prim, t, _, _ = trace(build(tris, **kw), rays)
    h = orc.brute(tris, rays)
    np.testing.assert_array_equal(prim, h.prim)
    np.testing.assert_array_equal(fbits(t), fbits(h.t))


@pytest.mark.gpu
@pytest.mark.parametrize("clustering", ["hploc", "ploc"])
def test_device_memory_limit_gives_out_of_memory_and_releases_everything(orc, limits, clustering):
    from gpu_util import build
    from diplodocus_b200 import scenes as S
    tris = S.soup(200_000, seed=9)
    rays = S.random_rays(2048, seed=9)
    import gc
    gc.collect()  # handles of earlier tests release their memory now, not during the measurement
    torch.cuda.synchronize()
    _, before = L.get_limits()
    limits(device_memory_bytes=before + (4 << 20))  # a build of 200k triangles needs far more than 4 MB
    with pytest.raises(L.DiplError) as e:
        build(tris, clustering=clustering)
    assert e.value.status == DIPL_ERR_OUT_OF_MEMORY and "limit" in str(e.value)
    torch.cuda.synchronize()
    assert L.get_limits()[1] == before  # everything the failed build took went back
    limits()
    _check_build_and_trace(orc, tris, rays, clustering=clustering)


@pytest.mark.gpu
@pytest.mark.parametrize("clustering", ["hploc", "ploc"])
def test_clustering_iteration_limit_gives_internal_error(orc, limits, clustering):
    from gpu_util import build
    from diplodocus_b200 import scenes as S
    tris = S.soup(20_000, seed=10)
    limits(clustering_iterations=1)  # every clustering of 20k triangles needs more than one iteration
    with pytest.raises(L.DiplError) as e:
        build(tris, clustering=clustering)
    assert e.value.status == DIPL_ERR_INTERNAL and "converge" in str(e.value)
    limits()
    _check_build_and_trace(orc, tris, S.random_rays(2048, seed=10), clustering=clustering)


@pytest.mark.gpu
@pytest.mark.parametrize("layout,bv", [("binary", "aabb"), ("binary", "sobb"), ("wide8_q8", "aabb")])
def test_trace_step_limit_is_recorded_and_reported(orc, limits, layout, bv):
    from gpu_util import build, trace
    from diplodocus_b200 import accel as A
    from diplodocus_b200 import scenes as S
    kind = A.AccelerationStructureType.kPlocSobb if bv == "sobb" else A.AccelerationStructureType.kPloc
    tris = S.soup(50_000, seed=12)
    rays = S.random_rays(4096, seed=12)
    bvh = build(tris, kind, layout=layout)
    limits(trace_steps=2)  # a soup of 50k triangles is deeper than two steps for most rays
    h = bvh.Intersect(A.Stats(), torch.from_numpy(rays))
    torch.cuda.synchronize()
    with pytest.raises(L.DiplError) as e:
        bvh.check_errors()
    assert e.value.status == DIPL_ERR_INTERNAL
    assert (h.prim.cpu().numpy() >= -1).all()  # every record was written: the rays finished with what they had
    bvh.check_errors()  # reported once, then cleared
    limits()
    prim, t, _, _ = trace(bvh, rays)
    np.testing.assert_array_equal(prim, orc.brute(tris, rays).prim)
