"""The GPU frontend (wavefront ray generation): the host restatement pinned to the workload generator on the
CPU, the device generators bit-exact against the restatement, and a whole frame against brute force."""
import numpy as np
import pytest
import torch

from diplodocus_b200 import scenes as S

CAMERAS = [
    dict(S.SMALL_CAMERA, width=512, height=512),
    dict(cam_pos=(0.3, -0.2, 2.5), cam_dir=(-0.1, 0.05, -1.0), cam_up=(0.0, 1.0, 0.1), fov=0.7, far=50.0,
         width=320, height=200),
]


def _cam_args(c):
    return (c["cam_pos"], c["cam_dir"], c["cam_up"], c["fov"], c["far"], c["width"], c["height"])


@pytest.mark.parametrize("cam", CAMERAS)
def test_oracle_pinhole_equals_the_workload_generator(orc, cam):
    """The restated pinhole generator reproduces scenes.pinhole_rays (the reference camera formula) bit for bit."""
    got = orc.pinhole_rays(*_cam_args(cam))
    want = S.pinhole_rays(cam["width"], cam["height"], cam["cam_pos"], cam["cam_dir"], cam["cam_up"], cam["fov"],
                          cam["far"])
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))


def test_oracle_bounce_rays_are_cosine_samples_on_the_incoming_side(orc):
    tris, rays = S.small_scene(seed=1, width=64, height=64)
    h = orc.brute(tris, rays)
    b = orc.bounce_rays(tris, rays, h.prim, h.t, seed=7)
    hit = h.prim >= 0
    assert hit.sum() > 1000
    # misses: a ray that hits nothing (tmax = 0 < tmin)
    assert (b[~hit, 7] == 0.0).all() and (b[~hit, 3] > 0).all()
    d = b[hit, 4:7].astype(np.float64)
    np.testing.assert_allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-6)
    tri = tris[h.prim[hit]].astype(np.float64)
    ng = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    ng /= np.linalg.norm(ng, axis=1, keepdims=True)
    din = rays[hit, 4:7].astype(np.float64)
    ng[(ng * din).sum(1) > 0] *= -1.0
    cos = (d * ng).sum(1)
    assert (cos >= -1e-6).all()                        # the hemisphere facing the incoming ray
    assert abs(cos.mean() - 2.0 / 3.0) < 0.02          # E[cos] of a cosine-weighted hemisphere is 2/3
    pos = rays[hit, 0:3].astype(np.float64) + din * h.t[hit, None]
    off = ((b[hit, 0:3] - pos) * ng).sum(1)
    assert (off > 0).all() and (off <= 1.1e-3).all()   # RayEpsilon offset along the facing normal
    # the same seed gives the same rays, another seed other directions
    np.testing.assert_array_equal(orc.bounce_rays(tris, rays, h.prim, h.t, seed=7), b)
    assert not np.array_equal(orc.bounce_rays(tris, rays, h.prim, h.t, seed=8)[hit], b[hit])


@pytest.mark.gpu
@pytest.mark.parametrize("cam", CAMERAS)
def test_device_pinhole_rays_bit_exact(orc, cam):
    from diplodocus_b200 import accel as A
    got = A.generate_pinhole_rays(*_cam_args(cam)).cpu().numpy()
    want = orc.pinhole_rays(*_cam_args(cam))
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [1, 12345])
def test_device_bounce_rays_bit_exact(orc, seed):
    from diplodocus_b200 import accel as A
    tris, rays = S.small_scene(seed=2, width=128, height=128)
    bvh = A.GpuPlocBvh().Build(A.AccelerationStructureConfig(), A.Stats(), torch.from_numpy(tris))
    dr = torch.from_numpy(rays).cuda()
    h = bvh.Intersect(A.Stats(), dr)
    got = A.generate_bounce_rays(bvh._v, dr, h, seed).cpu().numpy()
    want = orc.bounce_rays(tris, rays, h.prim.cpu().numpy(), h.t.cpu().numpy(), seed)
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.gpu
def test_frame_primary_and_bounce_hits_bit_exact_with_brute_force(orc):
    """generate -> trace -> bounce -> trace on the device: both hit sets equal the oracle's brute force."""
    from diplodocus_b200 import accel as A
    tris, _ = S.small_scene(seed=3, width=8, height=8)
    bvh = A.GpuPlocBvh().Build(A.AccelerationStructureConfig(), A.Stats(), torch.from_numpy(tris))
    rays, hits, bounce, bhits = A.trace_frame(bvh, dict(S.SMALL_CAMERA), 96, 96, seed=5)
    for r, h in ((rays, hits), (bounce, bhits)):
        ref = orc.brute(tris, r.cpu().numpy())
        np.testing.assert_array_equal(h.prim.cpu().numpy(), ref.prim)
        np.testing.assert_array_equal(h.t.cpu().numpy().view(np.uint32), ref.t.view(np.uint32))
    assert (bhits.prim >= 0).sum() > 100  # bounces inside the open box hit its walls


def test_generators_reject_bad_arguments():
    """No GPU needed: argument checks come before any device work."""
    import ctypes as C
    from diplodocus_b200 import _lib as L
    lib = L.load()
    cam = L.Camera((C.c_float * 3)(0, 0, 1), (C.c_float * 3)(0, 0, -1), (C.c_float * 3)(0, 1, 0), 0.9, 10.0)
    assert lib.dipl_generate_pinhole_rays(C.byref(cam), 1, 4, C.c_void_p(16), None) == 1  # DIPL_ERR_INVALID_ARGUMENT
    assert lib.dipl_generate_pinhole_rays(None, 4, 4, C.c_void_p(16), None) == 1  # DIPL_ERR_INVALID_ARGUMENT
    assert lib.dipl_generate_bounce_rays(None, None, None, None, None, 4, 0, None, None) == 1  # DIPL_ERR_INVALID_ARGUMENT
    assert lib.dipl_generate_bounce_rays(None, None, None, None, None, 0, 0, None, None) == L.DIPL_OK


# ---- the shadow wave (IsShadowed through dipl_bvh_trace_any) ---------------------------------------------------
def _lit_small_scene():
    """The small scene with two area lights (triangles of the box's top wall) and two point lights."""
    tris, _ = S.small_scene(seed=4, width=8, height=8)
    top = [i for i in range(10) if np.allclose(tris[i, :, 1], tris[i, 0, 1]) and tris[i, 0, 1] > 0.4]
    assert len(top) >= 2
    points = np.array([[0.0, 0.45, -0.2], [0.3, 0.2, 0.4]], np.float32)
    return tris, top[:2], points


def test_oracle_shadow_rays_follow_is_shadowed(orc):
    """Restated shadow rays: unit directions toward the light sample, origins offset by RayEpsilon on the light's
    side, tmax short of the light by RayEpsilon; null rays for misses and for hits on an area light."""
    tris, area, points = _lit_small_scene()
    rays = S.pinhole_rays(48, 48, **S.SMALL_CAMERA)
    h = orc.brute(tris, rays)
    sr = orc.shadow_rays(tris, rays, h.prim, h.t, 48, area, 3, points)
    per_hit = len(area) * 3 + len(points)
    assert sr.shape == (len(rays) * per_hit, 8)
    sr = sr.reshape(len(rays), per_hit, 8)
    miss = h.prim < 0
    assert (sr[miss, :, 7] == 0).all()
    for j, tri in enumerate(area):  # a hit on area light j: the reference returns its colour at light j, so
        on = h.prim == tri          # lights before j were sampled and j and later ones cast nothing
        assert on.any()
        assert (sr[on, j * 3: len(area) * 3, 7] == 0).all()
    cast = sr[:, :, 7] > 0
    assert cast.sum() > 1000
    d = sr[cast][:, 4:7].astype(np.float64)
    np.testing.assert_allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-6)
    # point-light rays end just short of the light
    pl = sr[~miss, len(area) * 3:, :]
    cast_pl = pl[:, :, 7] > 0
    end = pl[..., 0:3].astype(np.float64) + pl[..., 4:7] * pl[..., 7:8]
    for j, p in enumerate(points):
        gap = np.linalg.norm(end[:, j] - p, axis=1)[cast_pl[:, j]]
        assert (gap < 2e-3).all()


@pytest.mark.gpu
def test_device_shadow_wave_bit_exact(orc):
    """Device shadow rays equal the restatement bit for bit, and their occlusion (dipl_bvh_trace_any) equals the
    oracle's any-hit brute force (IntersectAny semantics: tmin < t < tmax)."""
    from diplodocus_b200 import accel as A
    tris, area, points = _lit_small_scene()
    bvh = A.GpuPlocBvh().Build(A.AccelerationStructureConfig(), A.Stats(), torch.from_numpy(tris))
    lights = A.Lights(area_light_triangles=tuple(area), samples=3, point_lights=tuple(map(tuple, points)))
    st = A.Stats()
    rays, hits, bounce, bhits, shadow, occ = A.trace_frame(bvh, dict(S.SMALL_CAMERA), 64, 64, seed=5, stats=st,
                                                           lights=lights)
    want = orc.shadow_rays(tris, rays.cpu().numpy(), hits.prim.cpu().numpy(), hits.t.cpu().numpy(), 64, area, 3,
                           points)
    got = shadow.cpu().numpy()
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))
    np.testing.assert_array_equal(occ.cpu().numpy(), orc.brute_any(tris, want))
    assert 0 < occ.cpu().numpy().sum() < (want[:, 7] > 0).sum()  # some shadowed, some lit
    assert st.rt_stats.shadow_ray_count == int((want[:, 7] > 0).sum())
