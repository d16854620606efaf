"""CPU: host-side mirror of the reference interface and the workload generators."""
import numpy as np
import pytest

from diplodocus_b200 import scenes as S


def test_parse_and_bridge():
    from diplodocus_b200 import accel as A
    assert A.parse_acceleration_structure_type("ploc_emc_sobb") is A.AccelerationStructureType.kPlocEmcSobb
    with pytest.raises(RuntimeError):
        A.parse_acceleration_structure_type("bvh2")
    with pytest.raises(ValueError):
        A.CreateAccelerationStucture(A.AccelerationStructureConfig(A.AccelerationStructureType.kSbvh))


def test_hash_matches_reference_formula():
    # HashU32 (src/util/util.h:24-32) on a few inputs, evaluated with Python ints
    def h(x):
        x &= 0xFFFFFFFF
        x ^= x >> 16
        x = (x * 0x7FEB352D) & 0xFFFFFFFF
        x ^= x >> 15
        x = (x * 0x846CA68B) & 0xFFFFFFFF
        x ^= x >> 16
        return x
    xs = np.array([0, 1, 2, 12345, 0xFFFFFFFF], np.uint32)
    assert [int(v) for v in S.hash_u32(xs)] == [h(int(v)) for v in xs]


def test_workload_sizes():
    tris, rays = S.small_scene(width=8, height=8)
    assert tris.shape == (10 + 3968, 3, 3) and rays.shape == (64, 8)
    assert S.uv_sphere(16, 8).shape[0] == 2 * 16 * 7
    # 1024x512 sphere = 1,046,528 triangles; 256x128 = 65,024
    assert 2 * 1024 * 511 == 1046528 and 2 * 256 * 127 == 65024
    sizes = S.batched_mesh_sizes()
    assert len(sizes) == 256
    n = [2 * a * (b - 1) for a, b in sizes]
    assert 900 <= min(n) and max(n) <= 2_100_000


def test_rays_are_unit_and_inward():
    r = S.sphere_inward_rays(1000, seed=1)
    d = r[:, 4:7].astype(np.float64)
    assert np.allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-6)
    assert ((r[:, 0:3] * r[:, 4:7]).sum(axis=1) <= 0).all()
    p = S.pinhole_rays(16, 16, **S.SMALL_CAMERA)
    assert np.allclose(np.linalg.norm(p[:, 4:7].astype(np.float64), axis=1), 1.0, atol=1e-6)


def test_soup_distribution():
    t = S.soup(20000, seed=5)
    e = np.linalg.norm(t[:, 1] - t[:, 0], axis=1)
    lg = np.log(e)
    assert -6.4 < np.median(lg) < -5.3
    c = t.mean(axis=1)
    assert (c > -0.01).all() and (c < 1.01).all()
