"""GPU: the batching and differentiation forms and the FP64 oracle re-intersection."""
import numpy as np
import pytest
import torch

from diplodocus_b200 import _lib as L
from diplodocus_b200 import accel as A
from diplodocus_b200 import scenes as S
from gpu_util import build, fbits, trace

pytestmark = pytest.mark.gpu


def test_batched_build_equals_individual_builds(orc):
    meshes = [S.uv_sphere(nu, nu // 2, 1.0, (0, 0, 0), displacement=0.05, seed=10 + i)
              for i, nu in enumerate((8, 24, 64, 16, 128, 40, 12, 96))]
    meshes.insert(3, np.zeros((0, 3, 3), np.float32))  # an empty mesh in the batch
    cfg = A.AccelerationStructureConfig()
    bvhs = A.build_batched(cfg, [torch.from_numpy(m) for m in meshes])
    for m, b in zip(meshes, bvhs):
        rays = S.sphere_inward_rays(2048, seed=len(m))
        ref = build(m)
        p0, t0, u0, v0 = trace(ref, rays)
        p1, t1, u1, v1 = trace(b, rays)
        np.testing.assert_array_equal(p1, p0)
        np.testing.assert_array_equal(fbits(t1), fbits(t0))
        if len(m):
            assert b.sah_cost() == pytest.approx(ref.sah_cost(), rel=1e-9)


def test_batched_build_many_meshes_against_brute_force(orc):
    meshes = [S.soup(n, seed=n) for n in (1, 2, 3, 7, 50, 400, 3000, 9000)]
    bvhs = A.build_batched(A.AccelerationStructureConfig(A.AccelerationStructureType.kPlocEmc),
                           [torch.from_numpy(m) for m in meshes])
    for m, b in zip(meshes, bvhs):
        rays = S.random_rays(1024, seed=len(m))
        p, t, _, _ = trace(b, rays)
        h = orc.brute(m, rays)
        np.testing.assert_array_equal(p, h.prim)
        np.testing.assert_array_equal(fbits(t), fbits(h.t))


def test_reintersect_f64_matches_oracle(orc):
    tris, rays = S.small_scene(seed=2, width=64, height=64)
    bvh = build(tris)
    h = bvh.Intersect(A.Stats(), torch.from_numpy(rays))
    tuv = A.reintersect_f64(bvh._v, torch.from_numpy(rays).cuda(), h).cpu().numpy()
    prim = h.prim.cpu().numpy()
    t64, u64, v64 = orc.intersect_f64(tris, rays, prim)
    hit = prim >= 0
    np.testing.assert_allclose(tuv[hit, 0], t64[hit], rtol=1e-12)
    np.testing.assert_allclose(tuv[hit, 1], u64[hit], rtol=1e-9, atol=1e-12)
    # FP32 t of the reference-exact test against the FP64 oracle: relative error stays small
    t32 = h.t.cpu().numpy()[hit].astype(np.float64)
    assert np.max(np.abs(t32 - t64[hit]) / t64[hit]) < 1e-4


def _tuv64(T, O, D):
    """FP64 (t, u, v) of rays O + t D against triangles T (K, 3, 3): the closest-hit system solved by Cramer's rule
    (the Moller-Trumbore algebra of src/scene/triangle.cc:10-43 without its culling)."""
    a, b, c = T[:, 0], T[:, 1], T[:, 2]
    e1, e2, s = b - a, c - a, O - a
    p = np.cross(D, e2)
    det = (e1 * p).sum(1)
    q = np.cross(s, e1)
    return (e2 * q).sum(1) / det, (s * p).sum(1) / det, (D * q).sum(1) / det


@pytest.mark.parametrize("loss_kind", ["depth", "depth_and_barycentrics"])
def test_adjoint_matches_fp64_central_differences(loss_kind):
    """The differentiation configuration at full size: a 256x128 displaced sphere (65,024 triangles, indexed, so a
    mesh vertex is shared by up to six triangles) and 1024x1024 pinhole rays. Loss = sum over rays hitting both
    meshes of (t - t*)^2, and with "depth_and_barycentrics" also (u - u*)^2 + (v - v*)^2, where t*, u*, v* are
    the hits of a second, differently displaced sphere (the seeded target). The adjoint's gradients with respect
    to 1000 sampled mesh vertices and to 200 ray origins and directions are checked against FP64 central
    differences (h = 1e-4) of the same loss with the hit ids held fixed."""
    from diplodocus_b200.autograd import closest_hit_tuv
    verts, idx, rays = S.diff_scene()
    tverts, tidx = S.uv_sphere_indexed(256, 128, 1.0, (0.0, 0.0, 0.0), displacement=0.05, seed=6)
    assert len(idx) == 65024 and len(rays) == 1 << 20
    tris = verts[idx].astype(np.float32)
    bvh = build(tris)
    tp, tt, tu, tv = trace(build(tverts[tidx].astype(np.float32)), rays)
    V = torch.from_numpy(verts.astype(np.float32)).cuda().requires_grad_(True)
    it = torch.from_numpy(idx).cuda()
    v0, v1, v2 = (V[it[:, k]] for k in range(3))  # per-triangle corners gathered from the shared vertices
    o = torch.from_numpy(rays[:, 0:3].copy()).cuda().requires_grad_(True)
    d = torch.from_numpy(rays[:, 4:7].copy()).cuda().requires_grad_(True)
    t, u, v, prim = closest_hit_tuv(v0, v1, v2, o, d, bvh, tmax=100.0)
    prim_np = prim.cpu().numpy()
    sel = (prim_np >= 0) & (tp >= 0)
    assert sel.sum() > 200_000
    w_uv = 1.0 if loss_kind == "depth_and_barycentrics" else 0.0
    m = torch.from_numpy(sel).cuda()
    tgt = [torch.from_numpy(x.astype(np.float32)).cuda() for x in (tt, tu, tv)]
    zero = torch.zeros_like(t)
    loss = (torch.where(m, (t - tgt[0]) ** 2, zero).sum()
            + w_uv * torch.where(m, (u - tgt[1]) ** 2 + (v - tgt[2]) ** 2, zero).sum())
    loss.backward()
    gV = V.grad.detach().cpu().numpy().astype(np.float64)
    go = o.grad.detach().cpu().numpy().astype(np.float64)
    gd = d.grad.detach().cpu().numpy().astype(np.float64)

    # FP64 oracle. Only the rays that hit a triangle touching the perturbed vertex change, so each difference is
    # taken over those rays (the other terms cancel exactly).
    Vd = verts.astype(np.float32).astype(np.float64)
    R = rays.astype(np.float64)
    T64 = (tt.astype(np.float64), tu.astype(np.float64), tv.astype(np.float64))
    rays_sel = np.nonzero(sel)[0]
    order = np.argsort(prim_np[rays_sel], kind="stable")
    by_tri = rays_sel[order]
    starts = np.searchsorted(prim_np[by_tri], np.arange(len(idx) + 1))
    tris_of_vertex = [[] for _ in range(len(verts))]
    for tri, corners in enumerate(idx):
        for c in corners:
            tris_of_vertex[c].append(tri)

    def loss_terms(Vm, ray_ids):
        T = Vm[idx[prim_np[ray_ids]]]
        t64, u64, v64 = _tuv64(T, R[ray_ids, 0:3], R[ray_ids, 4:7])
        out = (t64 - T64[0][ray_ids]) ** 2
        if w_uv:
            out = out + (u64 - T64[1][ray_ids]) ** 2 + (v64 - T64[2][ray_ids]) ** 2
        return out.sum()

    rng = np.random.default_rng(7)
    hit_vertices = np.unique(idx[np.unique(prim_np[rays_sel])])
    h = 1e-4
    errs = []
    for vert in rng.choice(hit_vertices, 1000, replace=False):
        ray_ids = np.concatenate([by_tri[starts[tri]:starts[tri + 1]] for tri in tris_of_vertex[vert]])
        a = int(rng.integers(0, 3))
        Vp, Vm = Vd.copy(), Vd.copy()
        Vp[vert, a] += h
        Vm[vert, a] -= h
        fd = (loss_terms(Vp, ray_ids) - loss_terms(Vm, ray_ids)) / (2 * h)
        errs.append(abs(gV[vert, a] - fd) / max(abs(fd), 1e-3))
    errs = np.array(errs)
    assert np.median(errs) < 1e-3 and np.quantile(errs, 0.95) < 2e-2, (np.median(errs), np.quantile(errs, 0.95))

    def ray_loss(Rm, ray):
        T = Vd[idx[prim_np[ray]]][None]
        t64, u64, v64 = _tuv64(T, Rm[None, 0:3], Rm[None, 4:7])
        out = (t64[0] - T64[0][ray]) ** 2
        if w_uv:
            out += (u64[0] - T64[1][ray]) ** 2 + (v64[0] - T64[2][ray]) ** 2
        return out

    rerr = []
    for ray in rng.choice(rays_sel, 200, replace=False):
        for col, grad in ((0, go), (4, gd)):
            a = int(rng.integers(0, 3))
            Rp, Rm = R[ray].copy(), R[ray].copy()
            Rp[col + a] += h
            Rm[col + a] -= h
            fd = (ray_loss(Rp, ray) - ray_loss(Rm, ray)) / (2 * h)
            rerr.append(abs(grad[ray, a] - fd) / max(abs(fd), 1e-3))
    rerr = np.array(rerr)
    assert np.median(rerr) < 1e-3 and np.quantile(rerr, 0.95) < 2e-2, (np.median(rerr), np.quantile(rerr, 0.95))
    # rays outside the loss get no gradient
    assert np.all(go[~sel] == 0.0) and np.all(gd[~sel] == 0.0)


def test_build_plan_graph_replay_matches_fresh_builds(orc):
    """The graph-captured batch rebuilds from the current vertices: equal to fresh builds before and after a
    deformation of the vertex arrays."""
    meshes = [S.uv_sphere(nu, nu // 2, 1.0, (0, 0, 0), displacement=0.05, seed=30 + i)
              for i, nu in enumerate((16, 64, 40, 128))] + [S.soup(3000, seed=9)]
    for kind in (A.AccelerationStructureType.kPloc, A.AccelerationStructureType.kPlocEmcSobb):
        cfg = A.AccelerationStructureConfig(kind)
        plan = A.BuildPlan(cfg, [torch.from_numpy(m) for m in meshes])
        for step in range(2):
            if step == 1:  # deform in place: the plan holds the same device arrays
                for v in plan.verts:
                    for x in v:
                        x.mul_(1.1).add_(0.01)
            plan.launch()
            bvhs = plan.bvhs()
            for i, b in enumerate(bvhs):
                tris_now = torch.stack([x for x in plan.verts[i]], dim=1).cpu().numpy()
                rays = S.sphere_inward_rays(1024, seed=i) if i < 4 else S.random_rays(1024, seed=i)
                p1, t1, _, _ = trace(b, rays)
                h = orc.brute(tris_now, rays)
                np.testing.assert_array_equal(p1, h.prim)
                np.testing.assert_array_equal(fbits(t1), fbits(h.t))
        plan.close()


def test_autotuner_picks_valid_knobs_and_caches(tmp_path):
    meshes = [torch.from_numpy(S.uv_sphere(256, 128, 1.0, (0, 0, 0), displacement=0.05, seed=3))]
    cfg = A.AccelerationStructureConfig()
    cache = str(tmp_path / "tune.jsonl")
    tuned, from_cache, _ = A.autotune(cfg, meshes, cache)
    assert not from_cache
    d = tuned[0]
    assert d.nn_search_radius in (8, 12, 16, 24, 32) and d.ploc_block_size in (128, 256, 512)
    assert d.sort_digit_bits in (6, 8, 10)
    tuned2, from_cache2, _ = A.autotune(cfg, meshes, cache)
    assert from_cache2 and tuned2[0].nn_search_radius == d.nn_search_radius
    assert '"key": "morton30/aabb/binary/L4/hploc/b' in open(cache).read()


@pytest.mark.parametrize("clustering", ["hploc", "ploc"])
def test_autotuned_build_keeps_the_sah_rule_and_is_not_slower(tmp_path, clustering):
    """The tuned knobs build a tree whose SAH cost is within 2% of the radius-16 default's (the tuner's rule) and
    the tuned build is not slower than the default beyond timing noise."""
    import time
    meshes = [torch.from_numpy(S.uv_sphere(nu, nu // 2, 1.0, (0, 0, 0), displacement=0.05, seed=nu))
              for nu in (64, 200, 512)]
    cfg = A.AccelerationStructureConfig(clustering=clustering)
    tuned, _, _ = A.autotune(cfg, meshes, str(tmp_path / "tune.jsonl"))
    default = A.AccelerationStructureConfig(clustering=clustering)

    def run(desc_fix):
        best, costs = 1e30, None
        for _ in range(5):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            bvhs = A.build_batched(desc_fix, meshes)
            torch.cuda.synchronize()
            best = min(best, time.perf_counter() - t0)
            costs = [b.sah_cost() for b in bvhs]
        return best, costs

    t_def, c_def = run(default)
    d0 = tuned[0]
    tuned_clustering = "ploc" if d0.clustering == L.CLUSTER_PLOC else "hploc"  # the tuner may switch it
    tcfg = A.AccelerationStructureConfig(clustering=tuned_clustering, nn_search_radius=d0.nn_search_radius,
                                         ploc_block_size=d0.ploc_block_size, sort_digit_bits=d0.sort_digit_bits)
    t_tun, c_tun = run(tcfg)
    w = np.array([len(m) for m in meshes], np.float64)
    assert np.dot(c_tun, w) / w.sum() <= 1.02 * np.dot(c_def, w) / w.sum()
    assert t_tun <= 1.25 * t_def, (t_tun, t_def)
