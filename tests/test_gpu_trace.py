"""GPU: closest-hit parity against the reference's own answers (golden fixtures) and the oracle."""
import numpy as np
import pytest
import torch

from conftest import GOLDEN_NAMES, load_golden
from diplodocus_b200 import accel as A
from diplodocus_b200 import scenes as S
from gpu_util import build, fbits, trace

pytestmark = pytest.mark.gpu

KINDS = [A.AccelerationStructureType.kPloc, A.AccelerationStructureType.kPlocEmc]


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_ref_mt_hits_bit_exact_with_reference_brute_force(name, kind):
    """Class E/T of the parity protocol: id, t, u, v bit-equal to DummyAccelerationStucture::Intersect."""
    g = load_golden(name)
    bvh = build(g["tris"], kind)
    prim, t, u, v = trace(bvh, g["rays"], leaf_test="ref_mt")
    np.testing.assert_array_equal(prim, g["brute_prim"])
    np.testing.assert_array_equal(fbits(t), fbits(g["brute_t"]))
    np.testing.assert_array_equal(fbits(u), fbits(g["brute_u"]))
    np.testing.assert_array_equal(fbits(v), fbits(g["brute_v"]))


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_agreement_classes_against_reference_sbvh(name):
    """Every ray where the GPU and the reference SBvh differ is an SBvh miss proven by brute force (class S)."""
    g = load_golden(name)
    prim, t, _, _ = trace(build(g["tris"]), g["rays"])
    diff = prim != g["sbvh_prim"]
    # the GPU answer is the brute-force answer on every ray ...
    np.testing.assert_array_equal(prim[diff], g["brute_prim"][diff])
    # ... and where SBvh differs it either missed the hit, took a farther one, or broke an exact tie by order
    sb_t = np.where(g["sbvh_prim"] >= 0, g["sbvh_t"], np.inf)
    assert (sb_t[diff] >= t[diff]).all()


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_watertight_matches_restatement(orc, name):
    g = load_golden(name)
    prim, t, u, v = trace(build(g["tris"]), g["rays"], leaf_test="watertight")
    h = orc.brute(g["tris"], g["rays"], leaf_test=1)
    np.testing.assert_array_equal(prim, h.prim)
    np.testing.assert_array_equal(fbits(t), fbits(h.t))
    np.testing.assert_array_equal(fbits(u), fbits(h.u))
    np.testing.assert_array_equal(fbits(v), fbits(h.v))


@pytest.mark.parametrize("leaf_test", [0, 1])
def test_backface_culling(orc, leaf_test):
    g = load_golden("small_scene")
    prim, t, _, _ = trace(build(g["tris"]), g["rays"], backface_culling=True,
                          leaf_test=["ref_mt", "watertight"][leaf_test])
    h = orc.brute(g["tris"], g["rays"], leaf_test=leaf_test, backface=True)
    np.testing.assert_array_equal(prim, h.prim)
    np.testing.assert_array_equal(fbits(t), fbits(h.t))


@pytest.mark.parametrize("name", ["small_scene", "soup_2k", "duplicates_ties"])
def test_any_hit_matches_oracle(orc, name):
    g = load_golden(name)
    rays = g["rays"].copy()
    rays[:, 7] = np.where(np.arange(len(rays)) % 2 == 0, rays[:, 7], 0.5)  # half the rays: short shadow rays
    bvh = build(g["tris"])
    occ = bvh.IntersectAny(A.Stats(), torch.from_numpy(rays)).cpu().numpy()
    np.testing.assert_array_equal(occ, orc.brute_any(g["tris"], rays))


@pytest.mark.parametrize("leaf", [2, 3, 5, 8])
def test_leaf_sizes(orc, leaf):
    g = load_golden("small_scene_full_mesh")
    prim, t, _, _ = trace(build(g["tris"], max_triangles_per_leaf=leaf), g["rays"])
    np.testing.assert_array_equal(prim, g["brute_prim"])


@pytest.mark.parametrize("radius", [1, 8, 32])
@pytest.mark.parametrize("block", [128, 256, 512])
def test_radius_and_block_size(radius, block):
    g = load_golden("soup_2k")
    prim, t, _, _ = trace(build(g["tris"], nn_search_radius=radius, ploc_block_size=block), g["rays"])
    np.testing.assert_array_equal(prim, g["brute_prim"])


def test_empty_scene_and_tiny_scenes(orc):
    rays = S.random_rays(256, seed=1)
    prim, t, _, _ = trace(build(np.zeros((0, 3, 3), np.float32)), rays)
    assert (prim == -1).all() and np.isinf(t).all()
    for n in (1, 2, 3, 4, 5):
        tris = S.soup(n, seed=n)
        tris = (tris - tris.mean(axis=(0, 1))) * 50 + 0.5  # large enough to be hit
        h = orc.brute(tris, rays)
        prim, t, _, _ = trace(build(tris), rays)
        np.testing.assert_array_equal(prim, h.prim)
        np.testing.assert_array_equal(fbits(t), fbits(h.t))


def test_axis_parallel_rays_and_rays_on_box_planes(orc):
    tris = S.open_box()
    o = np.array([[0.0, 0.0, 0.0], [0.5, 0.0, 0.0], [-0.5, 0.2, 0.1], [0.0, 0.5, 0.3], [0.1, -0.2, 0.4]], np.float32)
    d = np.array([[1, 0, 0], [0, 1, 0], [0, 0, -1], [-1, 0, 0], [0, -1, 0], [0, 0, 1]], np.float32)
    oo = np.repeat(o, len(d), axis=0)
    dd = np.tile(d, (len(o), 1))
    rays = S.pack_rays(oo, dd)
    h = orc.brute(tris, rays)
    prim, t, _, _ = trace(build(tris, max_triangles_per_leaf=2), rays)
    np.testing.assert_array_equal(prim, h.prim)


def test_counted_trace_counts():
    g = load_golden("displaced_sphere_64x32")
    bvh = build(g["tris"])
    st = A.Stats()
    bvh.Intersect(st, torch.from_numpy(g["rays"]), count=True)
    assert st.accel_stats.traversal_count > 0 and st.accel_stats.intersection_count > 0
    assert st.accel_stats.query_count == len(g["rays"])


def test_displaced_sphere_1m_hits_verified(orc):
    """Full size (1,046,528 triangles): every reported hit re-tests bit-exactly; a ray sample is
    bit-exact against the brute-force oracle (closest hit, lowest-id ties)."""
    tris, rays = S.displaced_sphere(n_rays=1 << 20)
    bvh = build(tris)
    prim, t, u, v = trace(bvh, rays)
    hit = prim >= 0
    assert 0.02 < hit.mean() < 0.2
    re = orc.test_pairs(tris, rays[hit], prim[hit])
    np.testing.assert_array_equal(fbits(re.t), fbits(t[hit]))
    np.testing.assert_array_equal(fbits(re.u), fbits(u[hit]))
    sample = np.concatenate([np.nonzero(hit)[0][:384], np.nonzero(~hit)[0][:128]])
    h = orc.brute(tris, rays[sample])
    np.testing.assert_array_equal(prim[sample], h.prim)
    np.testing.assert_array_equal(fbits(t[sample]), fbits(h.t))
