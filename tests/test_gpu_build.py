"""GPU: codes, sort and PLOC topology against the oracle, bit for bit."""
import numpy as np
import pytest
import torch

import oracle as O
from diplodocus_b200 import _lib as L
from diplodocus_b200 import accel as A
from diplodocus_b200 import scenes as S
from gpu_util import build

pytestmark = pytest.mark.gpu


def _meshes():
    return {
        "small_scene": S.small_scene(width=4, height=4)[0],
        "soup_50k": S.soup(50000, seed=11),
        "sphere_128x64": S.uv_sphere(128, 64, 1.0, (0, 0, 0), displacement=0.05, seed=2),
        "duplicates": np.repeat(S.open_box(), 300, axis=0),
    }


@pytest.mark.parametrize("name", list(_meshes()))
def test_morton30_codes_match_oracle(orc, name):
    tris = _meshes()[name]
    got = A.compute_codes(tris, L.CODE_MORTON30).cpu().numpy().view(np.uint32)
    np.testing.assert_array_equal(got, orc.morton30(tris))


@pytest.mark.parametrize("name", list(_meshes()))
def test_emc60_codes_match_oracle(orc, name):
    tris = _meshes()[name]
    got = A.compute_codes(tris, L.CODE_EMC60).cpu().numpy().view(np.uint64)
    np.testing.assert_array_equal(got, orc.emc60(tris))


@pytest.mark.parametrize("n", [1, 2, 3839, 3840, 3841, 100_003, 1 << 20])
@pytest.mark.parametrize("key_bytes,end_bit", [(4, 30), (4, 32), (8, 60), (8, 64)])
def test_radix_sort_matches_stable_argsort(n, key_bytes, end_bit):
    rng = np.random.default_rng(n + end_bit)
    dt = np.uint32 if key_bytes == 4 else np.uint64
    hi = (1 << min(end_bit, 63)) - 1
    keys = rng.integers(0, hi, size=n, dtype=np.uint64).astype(dt)
    keys[: n // 3] = keys[0]  # many duplicates: stability matters
    kt = torch.from_numpy(keys.view(np.int32 if key_bytes == 4 else np.int64)).cuda()
    ko, vo = A.radix_sort_pairs(kt, None, 0, end_bit)
    mask = dt(hi) if end_bit < 64 else np.iinfo(dt).max
    order = np.argsort(keys & mask, kind="stable")
    np.testing.assert_array_equal(vo.cpu().numpy(), order.astype(np.int32))
    np.testing.assert_array_equal(ko.cpu().numpy().view(dt), keys[order])


@pytest.mark.parametrize("digit_bits", [6, 7, 8, 10])
def test_radix_sort_digit_widths(digit_bits):
    rng = np.random.default_rng(digit_bits)
    keys = rng.integers(0, 1 << 30, size=200_000, dtype=np.uint32)
    ko, vo = A.radix_sort_pairs(torch.from_numpy(keys.view(np.int32)).cuda(), None, 0, 30, digit_bits)
    np.testing.assert_array_equal(vo.cpu().numpy(), np.argsort(keys, kind="stable").astype(np.int32))


def test_radix_sort_rejects_bad_arguments():
    k = torch.zeros(4, dtype=torch.int32, device="cuda")
    with pytest.raises(L.DiplError):
        A.radix_sort_pairs(k, None, 0, 40)
    with pytest.raises(L.DiplError):
        A.radix_sort_pairs(k, None, 0, 32, 9)


CLUSTERINGS = ["hploc", "ploc"]


def _expected_topology(orc, tris, codes, perm, clustering, radius=16):
    """The restatement of the clustering the device ran: (children, boxes, iterations) by internal node id."""
    if clustering == "ploc":
        return orc.ploc(tris, perm, radius=radius)
    return orc.hploc(tris, perm, np.asarray(codes)[perm], radius=radius)


@pytest.mark.parametrize("clustering", CLUSTERINGS)
@pytest.mark.parametrize("n", [1, 2, 3, 5, 16, 17, 31, 32, 33, 1000, 1025, 4097, 30000])
@pytest.mark.parametrize("radius", [1, 4, 16, 32])
def test_ploc_topology_matches_oracle(orc, n, radius, clustering):
    tris = S.soup(n, seed=100 + n)
    bvh = build(tris, nn_search_radius=radius, clustering=clustering)
    perm, ch, bx = bvh.download_topology()
    codes = orc.morton30(tris)
    exp_perm = O.sort_perm(codes)
    np.testing.assert_array_equal(perm, exp_perm)
    if n < 2:
        return
    ech, ebx, it = _expected_topology(orc, tris, codes, exp_perm, clustering, radius)
    np.testing.assert_array_equal(ch, ech)
    np.testing.assert_array_equal(bx.view(np.uint32), ebx.view(np.uint32))
    assert bvh.info().ploc_iterations == it


@pytest.mark.parametrize("clustering", CLUSTERINGS)
@pytest.mark.parametrize("kind", [A.AccelerationStructureType.kPloc, A.AccelerationStructureType.kPlocEmc])
def test_ploc_topology_duplicates_and_emc(orc, kind, clustering):
    tris = np.concatenate([np.repeat(S.open_box(), 200, axis=0), S.soup(3000, seed=4)])
    bvh = build(tris, kind, clustering=clustering)
    perm, ch, bx = bvh.download_topology()
    codes = orc.morton30(tris) if kind is A.AccelerationStructureType.kPloc else orc.emc60(tris)
    exp_perm = O.sort_perm(codes)
    np.testing.assert_array_equal(perm, exp_perm)
    ech, ebx, it = _expected_topology(orc, tris, codes, exp_perm, clustering)
    np.testing.assert_array_equal(ch, ech)
    np.testing.assert_array_equal(bx.view(np.uint32), ebx.view(np.uint32))


@pytest.mark.parametrize("clustering", CLUSTERINGS)
@pytest.mark.parametrize("kind", [A.AccelerationStructureType.kPloc, A.AccelerationStructureType.kPlocEmc])
def test_ploc_topology_with_non_finite_triangles(orc, kind, clustering):
    """Triangles with NaN or infinite coordinates (never hittable) get empty boxes and stay out of the scene
    bounds on the device exactly as in the restatement: same codes, same topology, same boxes."""
    tris = S.soup(5000, seed=21).copy()
    rng = np.random.default_rng(3)
    bad = rng.choice(len(tris), 300, replace=False)
    for k, i in enumerate(bad):
        tris[i, rng.integers(3), rng.integers(3)] = [np.nan, np.inf, -np.inf][k % 3]
    tris[bad[:20]] = np.nan
    bvh = build(tris, kind, clustering=clustering)
    perm, ch, bx = bvh.download_topology()
    codes = orc.morton30(tris) if kind is A.AccelerationStructureType.kPloc else orc.emc60(tris)
    exp_perm = O.sort_perm(codes)
    np.testing.assert_array_equal(perm, exp_perm)
    ech, ebx, it = _expected_topology(orc, tris, codes, exp_perm, clustering)
    np.testing.assert_array_equal(ch, ech)
    np.testing.assert_array_equal(bx.view(np.uint32), ebx.view(np.uint32))
    assert np.isfinite(ebx[~np.isinf(ebx).all(axis=1)]).all()


@pytest.mark.parametrize("clustering", CLUSTERINGS)
def test_ploc_topology_1m_displaced_sphere(orc, clustering):
    tris = S.uv_sphere(1024, 512, 1.0, (0, 0, 0), displacement=0.05, seed=2)
    bvh = build(tris, clustering=clustering)
    perm, ch, bx = bvh.download_topology()
    codes = orc.morton30(tris)
    exp_perm = O.sort_perm(codes)
    np.testing.assert_array_equal(perm, exp_perm)
    ech, ebx, it = _expected_topology(orc, tris, codes, exp_perm, clustering)
    np.testing.assert_array_equal(ch, ech)
    assert bvh.info().ploc_iterations == it


@pytest.mark.parametrize("clustering", CLUSTERINGS)
def test_sah_cost_matches_oracle_on_same_topology(orc, clustering):
    tris = S.soup(20000, seed=21)
    bvh = build(tris, clustering=clustering)
    perm, ch, bx = bvh.download_topology()
    leaf_boxes = np.concatenate([tris[perm].min(axis=1), tris[perm].max(axis=1)], axis=1)
    expect = O.sah_cost_binary(ch, bx, len(tris), leaf_boxes, 4)
    assert bvh.sah_cost() == pytest.approx(expect, rel=1e-9)


def test_hierarchical_clustering_sah_close_to_global_ploc(orc):
    """The hierarchical clustering's tree costs about what the global PLOC loop's does (same distance, same tie
    rule, merges confined to radix-tree nodes): within 2% on a soup and on a displaced sphere."""
    for tris in (S.soup(200_000, seed=8), S.uv_sphere(256, 128, 1.0, (0, 0, 0), displacement=0.05, seed=2)):
        costs = [build(tris, clustering=c).sah_cost() for c in CLUSTERINGS]
        assert costs[0] == pytest.approx(costs[1], rel=0.02), costs


def test_build_rejects_bad_options():
    tris = S.soup(10, seed=1)
    for kw in (dict(nn_search_radius=0), dict(nn_search_radius=33), dict(max_triangles_per_leaf=1),
               dict(ploc_block_size=100), dict(sort_digit_bits=9)):
        with pytest.raises(L.DiplError):
            build(tris, **kw)


def test_empty_and_tiny_builds():
    for n in (0, 1, 2, 3):
        tris = S.soup(max(n, 1), seed=3)[:n]
        bvh = build(tris)
        info = bvh.info()
        assert info.num_triangles == n


@pytest.mark.parametrize("kind", [A.AccelerationStructureType.kPloc, A.AccelerationStructureType.kPlocEmc])
@pytest.mark.parametrize("budget", [20, 100])
def test_presplit_topology_matches_oracle(orc, kind, budget):
    """Pre-splitting: the device's pieces, their codes, sort and hierarchical clustering equal the restatement bit
    for bit (leaf order by triangle, every internal node's children and box)."""
    tris = np.concatenate([S.soup(30000, seed=41), S.soup(5, seed=42) * 40.0])  # a few very large triangles too
    bvh = build(tris, kind, split_budget=budget)
    perm, ch, bx = bvh.download_topology()
    pieces, ref_tri, rbox = orc.presplit(tris, budget)
    code = 0 if kind is A.AccelerationStructureType.kPloc else 1
    codes = orc.ref_codes(tris, pieces, ref_tri, rbox, code)
    order = np.argsort(codes, kind="stable")
    assert bvh.info().num_leaves == len(ref_tri) > len(tris)
    np.testing.assert_array_equal(perm, ref_tri[order])
    ech, ebx, it = orc.hploc_boxes(rbox[order], codes[order])
    np.testing.assert_array_equal(ch, ech)
    np.testing.assert_array_equal(bx.view(np.uint32), ebx.view(np.uint32))
    assert bvh.info().ploc_iterations == it


def test_presplit_changes_nothing_on_an_even_mesh():
    """No triangle of a displaced sphere is split: the build equals the one without pre-splitting."""
    tris = S.uv_sphere(256, 128, 1.0, (0, 0, 0), displacement=0.05, seed=2)
    a, b = build(tris), build(tris, split_budget=40)
    for x, y in zip(a.download_topology(), b.download_topology()):
        np.testing.assert_array_equal(x, y)


def test_presplit_rejected_in_build_plans():
    with pytest.raises(L.DiplError) as e:
        A.BuildPlan(A.AccelerationStructureConfig(split_budget=20), [torch.from_numpy(S.soup(100, seed=1))])
    assert e.value.status == 6  # DIPL_ERR_UNSUPPORTED
