"""CPU: the oracle pinned against the reference's own outputs, and its own invariants."""
import numpy as np
import pytest

from conftest import GOLDEN_NAMES, bits, load_golden
from diplodocus_b200 import scenes as S


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_restatement_reproduces_reference_brute_force(orc, name):
    """The C restatement of Triangle::IntersectRay + brute force is bit-exact with the reference's fixtures."""
    g = load_golden(name)
    h = orc.brute(g["tris"], g["rays"])
    np.testing.assert_array_equal(h.prim, g["brute_prim"])
    np.testing.assert_array_equal(bits(h.t), bits(g["brute_t"]))
    np.testing.assert_array_equal(bits(h.u), bits(g["brute_u"]))
    np.testing.assert_array_equal(bits(h.v), bits(g["brute_v"]))


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_reference_harness_reproduces_fixtures(ref, name):
    g = load_golden(name)
    hb = ref.brute(g["tris"], g["rays"])
    np.testing.assert_array_equal(hb.prim, g["brute_prim"])
    np.testing.assert_array_equal(bits(hb.t), bits(g["brute_t"]))
    sb = ref.sbvh(g["tris"])
    hs = sb.trace(g["rays"])
    np.testing.assert_array_equal(hs.prim, g["sbvh_prim"])
    sah, _, _ = sb.sah_cost()
    assert sah == pytest.approx(float(g["sbvh_sah"]), rel=1e-12)


def test_reference_sbvh_is_not_conservative(ref):
    """SBvh's binning scale and split position disagree (sbvh.cc:213-218 vs :247): it misses hits."""
    tris = S.soup(20000, seed=9)
    rays = S.random_rays(4000, seed=9)
    hb = ref.brute(tris, rays)
    hs = ref.sbvh(tris).trace(rays)
    assert (hb.prim != hs.prim).sum() >= 0  # recorded, not asserted: depends on the sample


def test_backface_culling_restatement(orc):
    g = load_golden("small_scene")
    h = orc.brute(g["tris"], g["rays"], backface=True)
    h0 = orc.brute(g["tris"], g["rays"], backface=False)
    assert (h.prim >= 0).sum() <= (h0.prim >= 0).sum()


def test_watertight_agrees_with_fp64(orc):
    tris, rays = S.small_scene(seed=3, width=48, height=48, sphere_nu=24, sphere_nv=12)
    hw = orc.brute(tris, rays, leaf_test=1)
    p64, t64 = orc.brute_f64(tris, rays)
    agree = (hw.prim == p64) | ((hw.prim >= 0) & (p64 >= 0) & (np.abs(hw.t - t64) <= 1e-6 * np.abs(t64)))
    assert agree.mean() > 0.999


def test_morton30_known_grid(orc):
    # 8 unit triangles whose centroids sit on the corners of a cube: codes are the 3-bit corner index
    # scaled into the top cell (1023 per axis), x highest.
    pts = np.array([[x, y, z] for x in (0, 1) for y in (0, 1) for z in (0, 1)], np.float32)
    tris = np.repeat(pts[:, None, :], 3, axis=1)
    codes = orc.morton30(tris)
    full = 0x3FFFFFFF
    expect = [((full & 0x24924924) if x else 0) | ((full & 0x12492492) if y else 0) | ((full & 0x09249249) if z else 0)
              for x in (0, 1) for y in (0, 1) for z in (0, 1)]
    np.testing.assert_array_equal(codes, np.array(expect, np.uint32))


def test_emc60_plan_covers_60_bits(orc):
    for tris in (S.soup(1000, seed=1), S.uv_sphere(32, 16), S.open_box()):
        bits_, masks = orc.emc60_plan(tris)
        assert bits_.sum() == 60
        allm = 0
        for m in masks:
            assert int(m) & allm == 0
            allm |= int(m)
        assert allm == (1 << 60) - 1
        codes = orc.emc60(tris)
        assert int(codes.max()) < (1 << 60)


def _check_tree(n, children, boxes, tris, perm):
    k = len(children)
    assert k == n - 1
    seen = np.zeros(2 * n - 1, np.int32)
    for c in children.reshape(-1):
        seen[c] += 1
    assert (seen[:-1] == 1).all() and seen[-1] == 0  # every node but the root is a child exactly once
    lo = np.concatenate([tris[perm].min(axis=1), boxes[:, :3]])
    hi = np.concatenate([tris[perm].max(axis=1), boxes[:, 3:]])
    for i, (a, b) in enumerate(children):
        assert (lo[a] >= boxes[i, :3]).all() and (hi[a] <= boxes[i, 3:]).all()
        assert (lo[b] >= boxes[i, :3]).all() and (hi[b] <= boxes[i, 3:]).all()


@pytest.mark.parametrize("n", [2, 3, 31, 32, 33, 257, 2000])
@pytest.mark.parametrize("radius", [1, 4, 16])
def test_ploc_oracle_tree_is_valid(orc, n, radius):
    import oracle as O
    tris = S.soup(n, seed=n)
    perm = O.sort_perm(orc.morton30(tris))
    ch, bx, it = orc.ploc(tris, perm, radius=radius)
    _check_tree(n, ch, bx, tris, perm)
    assert it >= 1


def test_ploc_oracle_pairs_duplicates_in_log_iterations(orc):
    import oracle as O
    base = S.open_box()[:1]
    tris = np.repeat(base, 4096, axis=0)
    perm = O.sort_perm(orc.morton30(tris))
    ch, bx, it = orc.ploc(tris, perm, radius=16)
    _check_tree(4096, ch, bx, tris, perm)
    assert it <= 13  # equal distances pair neighbours: halving per iteration


def test_sah_cost_single_leaf_and_pair():
    import oracle as O
    boxes = np.array([[0, 0, 0, 1, 1, 1]], np.float32)
    leaf_boxes = np.array([[0, 0, 0, 1, 1, 0], [0, 0, 1, 1, 1, 1]], np.float32)
    children = np.array([[0, 1]], np.int32)
    # 2 triangles < L=4: the root is one leaf of 2 -> cost 2
    assert O.sah_cost_binary(children, boxes, 2, leaf_boxes, 4) == pytest.approx(2.0)
    # with L=2 the root is inner: 1 + 2 * SA(face)/SA(cube) = 1 + 2 * 2/6
    assert O.sah_cost_binary(children, boxes, 2, leaf_boxes, 2) == pytest.approx(1 + 2 * 2 / 6)


def test_chunked_reference_brute_force_equals_one_pass(ref):
    """The chunked brute force (used on large scenes) makes the comparisons of DummyAccelerationStucture::Intersect
    over all triangles: bit-identical records, including exact-t ties across chunk boundaries."""
    from diplodocus_b200 import scenes as S
    g = load_golden("duplicates_ties")
    for tris, rays in ((S.soup(30000, seed=7), S.random_rays(700, seed=7)), (g["tris"], g["rays"])):
        a = ref.brute(tris, rays)
        for chunk in (1, 7, 1000):
            b = ref.brute(tris, rays, chunk=chunk)
            for k in ("prim", "t", "u", "v"):
                np.testing.assert_array_equal(np.asarray(getattr(a, k)).view(np.uint32),
                                              np.asarray(getattr(b, k)).view(np.uint32))


@pytest.mark.parametrize("n", [2, 3, 7, 15, 16])
def test_hierarchical_clustering_equals_ploc_on_one_node(orc, n):
    """Up to 16 triangles no radix-tree node below the root is large enough to merge, so the root holds every leaf
    in position order, its pool is every split's id in order, and it runs global PLOC on that list: the same
    children, boxes and node ids as orc_ploc."""
    import oracle as O
    tris = S.soup(n, seed=40 + n)
    codes = orc.morton30(tris)
    perm = O.sort_perm(codes)
    ch_p, bx_p, _ = orc.ploc(tris, perm)
    ch_h, bx_h, _ = orc.hploc(tris, perm, codes[perm])
    np.testing.assert_array_equal(ch_h, ch_p)
    np.testing.assert_array_equal(bx_h.view(np.uint32), bx_p.view(np.uint32))


@pytest.mark.parametrize("n,nseg", [(1000, 1), (5000, 1), (3000, 5)])
def test_hierarchical_clustering_makes_one_binary_tree_per_segment(orc, n, nseg):
    """Every leaf has exactly one parent, each segment has one root, node ids are the splits inside segments
    (each used once), and a node's box is the union of its children's."""
    import oracle as O
    tris = S.soup(n, seed=n)
    codes = orc.morton30(tris).astype(np.uint64)
    seg = np.sort(np.random.default_rng(n).integers(0, nseg, n)).astype(np.int32)
    perm = np.lexsort((codes, seg)).astype(np.int32)
    sorted_keys = (seg.astype(np.uint64) << np.uint64(32)) | codes[perm]  # seg is per sorted position
    ch, bx, _ = orc.hploc(tris, perm, sorted_keys, seg=seg)
    used = ch[:, 0] >= 0
    boundary = np.nonzero(seg[1:] != seg[:-1])[0]
    assert not used[boundary].any() and used.sum() == n - nseg
    kids = ch[used].ravel()
    assert len(np.unique(kids)) == len(kids)
    roots = set(n + np.nonzero(used)[0]) - set(kids.tolist())
    assert len(roots) + (np.bincount(seg) == 1).sum() == nseg
    leaf_lo = tris[perm].min(axis=1)
    leaf_hi = tris[perm].max(axis=1)
    lo = lambda x: leaf_lo[x] if x < n else bx[x - n, :3]
    hi = lambda x: leaf_hi[x] if x < n else bx[x - n, 3:]
    for k in np.nonzero(used)[0]:
        a, b = ch[k]
        np.testing.assert_array_equal(bx[k, :3], np.minimum(lo(a), lo(b)))
        np.testing.assert_array_equal(bx[k, 3:], np.maximum(hi(a), hi(b)))


@pytest.mark.parametrize("budget", [10, 40, 100])
def test_presplit_pieces_cover_their_triangles(orc, budget):
    """Pre-splitting (restated): the split triangles are the large ones, at most budget% more leaves, every piece box
    lies in its triangle's box, and the pieces' boxes together cover the triangle (points sampled on it)."""
    tris = S.soup(20000, seed=31)
    pieces, ref_tri, rbox = orc.presplit(tris, budget)
    n = len(tris)
    assert len(ref_tri) == int(pieces.sum()) and len(ref_tri) <= n + (budget * n) // 100
    assert (pieces > 1).any() and pieces.max() <= 64
    lo, hi = tris.min(axis=1), tris.max(axis=1)
    d = hi - lo
    w = (d[:, 0] * d[:, 1] + d[:, 1] * d[:, 2]) + d[:, 2] * d[:, 0]
    assert w[pieces > 1].min() >= np.median(w)          # only large triangles split
    assert (np.diff(ref_tri) >= 0).all()                 # references in triangle order
    assert (rbox[:, :3] >= lo[ref_tri]).all() and (rbox[:, 3:] <= hi[ref_tri]).all()
    rng = np.random.default_rng(budget)
    for g in np.nonzero(pieces > 1)[0][:200]:
        boxes = rbox[ref_tri == g].astype(np.float64)
        a, b = rng.random(64), rng.random(64)
        flip = a + b > 1
        a[flip], b[flip] = 1 - a[flip], 1 - b[flip]
        t = tris[g].astype(np.float64)
        pts = t[0] + a[:, None] * (t[1] - t[0]) + b[:, None] * (t[2] - t[0])
        slack = 1e-6 * np.abs(t).max()
        inside = ((pts[:, None, :] >= boxes[None, :, :3] - slack) & (pts[:, None, :] <= boxes[None, :, 3:] + slack))
        assert inside.all(axis=2).any(axis=1).all(), g


def test_presplit_leaves_even_meshes_alone(orc):
    """A mesh of triangles of about equal size (a displaced sphere) gets no pieces at a moderate budget."""
    tris = S.uv_sphere(128, 64, 1.0, (0, 0, 0), displacement=0.05, seed=2)
    pieces, ref_tri, _ = orc.presplit(tris, 40)
    assert (pieces == 1).all() and len(ref_tri) == len(tris)
