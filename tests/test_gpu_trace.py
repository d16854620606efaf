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


@pytest.mark.parametrize("split", [0, 60])
@pytest.mark.parametrize("layout", ["binary", "wide8_q8"])
@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_ref_mt_hits_bit_exact_with_reference_brute_force(name, kind, layout, split):
    """Class E/T of the parity protocol: id, t, u, v bit-equal to DummyAccelerationStucture::Intersect (also with
    large triangles pre-split: leaves hold whole triangles, so the records cannot change)."""
    g = load_golden(name)
    bvh = build(g["tris"], kind, layout=layout, split_budget=split)
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


@pytest.mark.parametrize("layout", ["binary", "wide8_q8"])
@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_watertight_matches_restatement(orc, name, layout):
    g = load_golden(name)
    prim, t, u, v = trace(build(g["tris"], layout=layout), g["rays"], leaf_test="watertight")
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


@pytest.mark.parametrize("layout", ["binary", "wide8_q8"])
@pytest.mark.parametrize("name", ["small_scene", "soup_2k", "duplicates_ties"])
def test_any_hit_matches_oracle(orc, name, layout):
    g = load_golden(name)
    rays = g["rays"].copy()
    rays[:, 7] = np.where(np.arange(len(rays)) % 2 == 0, rays[:, 7], 0.5)  # half the rays: short shadow rays
    bvh = build(g["tris"], layout=layout)
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


@pytest.mark.gpu
def test_long_grazing_rays_equal_brute_force(orc):
    """Rays that skim the displaced sphere take hundreds of steps. Traced first in a batch of 2^19 rays (the
    smallest batch that uses the offload), the warps whose chunks hold them hand their long rays to the
    warp-per-ray tail kernel. The first 2048 equal brute force (closest hit, lowest-id ties), and the counted
    trace returns the same records."""
    tris, rays = S.displaced_sphere(n_rays=1 << 20)
    o, d = rays[:, 0:3].astype(np.float64), rays[:, 4:7].astype(np.float64)
    closest = np.linalg.norm(np.cross(o, d), axis=1) / np.linalg.norm(d, axis=1)
    is_graze = (closest > 0.93) & (closest < 1.07)
    graze = rays[is_graze]
    assert len(graze) > 2048
    batch = np.ascontiguousarray(np.concatenate([graze, rays[~is_graze][: (1 << 19) - len(graze)]]))
    assert len(batch) == 1 << 19
    bvh = build(tris)
    prim, t, u, v = trace(bvh, batch)
    h = orc.brute(tris, graze[:2048])
    np.testing.assert_array_equal(prim[:2048], h.prim)
    np.testing.assert_array_equal(fbits(t[:2048]), fbits(h.t))
    np.testing.assert_array_equal(fbits(u[:2048]), fbits(h.u))
    st = A.Stats()
    hc = bvh.Intersect(st, torch.from_numpy(batch), count=True)
    np.testing.assert_array_equal(hc.prim.cpu().numpy(), prim)
    long = A.Stats()
    bvh.Intersect(long, torch.from_numpy(np.ascontiguousarray(graze[:2048])), count=True)
    assert long.accel_stats.traversal_count / 2048 > 20  # long rays indeed


def _decode_wide(nodes_bytes):
    """Numpy view of the 80-byte wide nodes and their decoded child boxes (FP32 fma emulated exactly)."""
    rec = np.frombuffer(nodes_bytes, dtype=np.dtype([
        ("p", "<f4", 3), ("e", "u1", 3), ("imask", "u1"), ("child_base", "<i4"), ("tri_base", "<i4"),
        ("meta", "u1", 8), ("qlo", "u1", (3, 8)), ("qhi", "u1", (3, 8))]))
    scale = np.ldexp(1.0, rec["e"].astype(np.int64) - 127)  # (M, 3)
    p = rec["p"].astype(np.float64)
    lo = (rec["qlo"] * scale[:, :, None] + p[:, :, None]).astype(np.float32)
    hi = (rec["qhi"] * scale[:, :, None] + p[:, :, None]).astype(np.float32)
    return rec, lo, hi


@pytest.mark.parametrize("name", ["small_scene_full_mesh", "soup_2k", "displaced_sphere_64x32"])
def test_wide_quantised_bounds_are_conservative(name):
    """Every triangle under a wide child slot lies inside that slot's decoded 8-bit box."""
    g = load_golden(name)
    bvh = build(g["tris"], layout="wide8_q8")
    nodes, tris, root = bvh.download_layout()
    rec, lo, hi = _decode_wide(nodes.tobytes())
    binfo = build(g["tris"]).info()
    assert bvh.info().node_bytes < binfo.node_bytes  # the compression the form exists for

    def subtree_tris(node):
        out = []
        r = rec[node]
        inner_rank = 0
        for k in range(8):
            if (r["imask"] >> k) & 1:
                out += subtree_tris(r["child_base"] + r["meta"][k])
            elif r["meta"][k]:
                first = r["tri_base"] + (r["meta"][k] & 31)
                out += list(range(first, first + (r["meta"][k] >> 5)))
        return out

    # the traversal finds an inner child from its slot alone: rank = inner slots below it; leaf triangles
    # of a node are packed in slot order
    for r in rec:
        toff = 0
        for k in range(8):
            if (r["imask"] >> k) & 1:
                assert r["meta"][k] == bin(int(r["imask"]) & ((1 << k) - 1)).count("1")
            elif r["meta"][k]:
                assert r["meta"][k] & 31 == toff
                toff += r["meta"][k] >> 5

    checked = 0
    for node in range(len(rec)):
        r = rec[node]
        for k in range(8):
            if (r["imask"] >> k) & 1:
                ids = subtree_tris(r["child_base"] + r["meta"][k])
            elif r["meta"][k]:
                first = r["tri_base"] + (r["meta"][k] & 31)
                ids = list(range(first, first + (r["meta"][k] >> 5)))
            else:
                continue
            v = tris[ids][:, :, :3].reshape(-1, 3)
            assert (v >= lo[node, :, k]).all() and (v <= hi[node, :, k]).all(), (node, k)
            checked += 1
            if checked > 3000:
                return


SOBB_KINDS = [A.AccelerationStructureType.kPlocSobb, A.AccelerationStructureType.kPlocEmcSobb]


@pytest.mark.parametrize("kind", SOBB_KINDS)
@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_sobb_hits_bit_exact_with_reference_brute_force(name, kind):
    g = load_golden(name)
    prim, t, u, v = trace(build(g["tris"], kind), g["rays"])
    np.testing.assert_array_equal(prim, g["brute_prim"])
    np.testing.assert_array_equal(fbits(t), fbits(g["brute_t"]))
    np.testing.assert_array_equal(fbits(u), fbits(g["brute_u"]))


@pytest.mark.parametrize("kdop", [6, 14, 26, 32])
def test_sobb_direction_sets(orc, kdop):
    g = load_golden("soup_2k")
    bvh = build(g["tris"], A.AccelerationStructureType.kPlocSobb, kdop_size=kdop)
    prim, t, _, _ = trace(bvh, g["rays"])
    np.testing.assert_array_equal(prim, g["brute_prim"])
    occ = bvh.IntersectAny(A.Stats(), torch.from_numpy(g["rays"])).cpu().numpy()
    np.testing.assert_array_equal(occ, orc.brute_any(g["tris"], g["rays"]))


SOBB_DIRS = np.array([
    [1, 0, 0], [0, 1, 0], [0, 0, 1],
    [0.57735026, 0.57735026, 0.57735026], [0.57735026, 0.57735026, -0.57735026],
    [0.57735026, -0.57735026, 0.57735026], [-0.57735026, 0.57735026, 0.57735026],
    [0.70710677, 0.70710677, 0], [0.70710677, -0.70710677, 0], [0.70710677, 0, 0.70710677],
    [0.70710677, 0, -0.70710677], [0, 0.70710677, 0.70710677], [0, 0.70710677, -0.70710677],
    [0, 0.52573111, 0.85065081], [0.52573111, 0.85065081, 0], [0.85065081, 0, 0.52573111]], np.float32)


@pytest.mark.parametrize("name", ["small_scene_full_mesh", "soup_2k"])
def test_sobb_slabs_contain_their_subtrees(name):
    """Every vertex under a child lies inside that child's three slabs (exact FP64 projections)."""
    g = load_golden(name)
    bvh = build(g["tris"], A.AccelerationStructureType.kPlocSobb)
    nodes, tris, root = bvh.download_layout()
    rec = np.frombuffer(nodes.tobytes(), dtype=np.dtype([("f", "<f4", 12), ("ref", "<i4", 2), ("ax", "<i4", 2)]))
    dirs = SOBB_DIRS.astype(np.float64)

    def leaf_range(ref):
        x = ~int(ref)
        return list(range(x >> 3, (x >> 3) + (x & 7)))

    def subtree(ref):
        if ref < 0:
            return leaf_range(ref)
        r = rec[ref]
        return subtree(r["ref"][0]) + subtree(r["ref"][1])

    n_checked = 0
    for k in range(len(rec)):
        f = rec[k]["f"]
        slabs = [(f[0:6], rec[k]["ax"][0]), (np.concatenate([f[6:12]]), rec[k]["ax"][1])]
        for side in range(2):
            vals, ax = slabs[side]
            ids = subtree(rec[k]["ref"][side])
            v = tris[ids][:, :, :3].reshape(-1, 3).astype(np.float64)
            for j in range(3):
                a = (int(ax) >> (8 * j)) & 0xFF
                pr = v @ dirs[a]
                assert (pr >= vals[2 * j]).all() and (pr <= vals[2 * j + 1]).all(), (k, side, j)
            n_checked += 1
        if n_checked > 2000:
            break
    assert n_checked > 0


@pytest.mark.parametrize("layout", ["binary", "wide8_q8"])
@pytest.mark.parametrize("kind", KINDS + SOBB_KINDS)
def test_nan_and_inf_vertices(orc, kind, layout):
    """Triangles with NaN or infinite coordinates neither fault the build nor hide valid geometry: every hit
    record equals the oracle's brute force bit for bit."""
    if layout == "wide8_q8" and kind in SOBB_KINDS:
        pytest.skip("the 8-wide layout has AABB children only")
    tris, rays = S.small_scene(seed=4, width=48, height=48)
    tris = tris.copy()
    rng = np.random.default_rng(9)
    bad = rng.choice(len(tris), 60, replace=False)
    for k, i in enumerate(bad):
        v, a = rng.integers(3), rng.integers(3)
        tris[i, v, a] = [np.nan, np.inf, -np.inf][k % 3]
    tris[bad[:3]] = np.nan  # a few triangles with no finite coordinate at all
    bvh = build(tris, kind, layout=layout)
    prim, t, u, v = trace(bvh, rays)
    ref = orc.brute(tris, rays)
    np.testing.assert_array_equal(prim, ref.prim)
    np.testing.assert_array_equal(fbits(t), fbits(ref.t))
    np.testing.assert_array_equal(fbits(u), fbits(ref.u))
    bvh.check_errors()


@pytest.mark.parametrize("form", ["binary", "sobb", "wide8_q8"])
@pytest.mark.parametrize("workload", ["sphere", "soup"])
def test_reordered_trace_equals_given_order(workload, form):
    """Batches of 2^20 rays or more are traced in a coherent order of their own; the records are bit-identical to
    tracing in the given order, in every layout. The visit and test totals agree to 0.1%: the binary trace hands
    long rays of nearly idle warps to the warp-per-ray tail kernel, which counts the nodes that warp visits, and
    which rays those are depends on the order."""
    if workload == "sphere":
        tris, rays = S.displaced_sphere(nu=256, nv=128, n_rays=1 << 20)
    else:
        tris, rays = S.soup(200_000, seed=5), S.random_rays((1 << 20) + 77, seed=5)
    kind = A.AccelerationStructureType.kPlocEmcSobb if form == "sobb" else A.AccelerationStructureType.kPlocEmc
    bvh = build(tris, kind, layout="wide8_q8" if form == "wide8_q8" else "binary")
    rd = torch.from_numpy(rays).cuda()
    st_a, st_b = A.Stats(), A.Stats()
    a = bvh.Intersect(st_a, rd, count=True)
    b = bvh.Intersect(st_b, rd, count=True, coherent_order=True)
    torch.cuda.synchronize()
    bvh.check_errors()
    assert torch.equal(a.raw, b.raw)
    for x, y in ((st_a.accel_stats.traversal_count, st_b.accel_stats.traversal_count),
                 (st_a.accel_stats.intersection_count, st_b.accel_stats.intersection_count)):
        assert abs(x - y) <= 1e-3 * max(x, y), (x, y)


@pytest.mark.parametrize("name", ["small_scene", "displaced_sphere_64x32", "soup_2k"])
@pytest.mark.parametrize("clustering", ["hploc", "ploc"])
def test_counted_trace_totals_equal_a_host_retraversal(orc, name, clustering):
    """The node-visit and triangle-test counters (the reference's traversal_count / intersection_count, sbvh.cc:76,83)
    equal a host re-traversal of the downloaded layout, ray for ray summed: the rays whose slab decisions are too
    close to call under the device's approximate reciprocal are left out of both sides."""
    g = load_golden(name)
    bvh = build(g["tris"], clustering=clustering)
    nodes, tris, root = bvh.download_layout()
    visits, tests, stable, prim, t = orc.retrace_binary(nodes, tris, root, g["rays"])
    assert stable.mean() > 0.95
    np.testing.assert_array_equal(prim[stable], g["brute_prim"][stable])  # the re-traversal is a correct trace
    st = A.Stats()
    bvh.Intersect(st, torch.from_numpy(np.ascontiguousarray(g["rays"][stable])), count=True)
    torch.cuda.synchronize()
    assert st.accel_stats.traversal_count == int(visits[stable].sum())
    assert st.accel_stats.intersection_count == int(tests[stable].sum())


@pytest.mark.parametrize("form", ["binary", "sobb", "wide8_q8"])
def test_presplit_hits_equal_brute_force_on_a_dense_soup(orc, form):
    """A soup at the 16M soup's density (200k triangles in a 0.31 cube: large triangles overlap everywhere), split
    at budget 40: every form's hits equal the brute force's bit for bit, and the rays visit fewer nodes and test
    fewer triangles than without splitting."""
    tris = S.soup(200_000, seed=44)
    c = tris.mean(axis=1, keepdims=True)
    tris = ((tris - c) + c * 0.31).astype(np.float32)
    rays = S.random_rays(8192, seed=44)
    rays[:, 0:3] *= 0.31
    kind = A.AccelerationStructureType.kPlocEmcSobb if form == "sobb" else A.AccelerationStructureType.kPlocEmc
    layout = "wide8_q8" if form == "wide8_q8" else "binary"
    h = orc.brute(tris, rays)
    counts = []
    for split in (0, 40):
        bvh = build(tris, kind, layout=layout, split_budget=split)
        prim, t, u, v = trace(bvh, rays)
        np.testing.assert_array_equal(prim, h.prim)
        np.testing.assert_array_equal(fbits(t), fbits(h.t))
        st = A.Stats()
        bvh.Intersect(st, torch.from_numpy(rays), count=True)
        counts.append((st.accel_stats.traversal_count, st.accel_stats.intersection_count))
    assert counts[1][0] < 0.8 * counts[0][0] and counts[1][1] < 0.6 * counts[0][1], counts
