"""GPU: the batching and differentiation forms and the FP64 oracle re-intersection."""
import numpy as np
import pytest
import torch

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


def test_adjoint_matches_fp64_central_differences():
    """dL/dvertex of L = sum (t - t_target)^2 against FP64 central differences (h = 1e-4) with hit ids fixed."""
    from diplodocus_b200.autograd import closest_hit_tuv
    verts, idx, rays = S.diff_scene(nu=64, nv=32, width=64, height=64)
    tris = verts[idx].astype(np.float32)
    bvh = build(tris)
    v0, v1, v2 = (torch.from_numpy(np.ascontiguousarray(tris[:, k])).cuda().requires_grad_(True) for k in range(3))
    o = torch.from_numpy(rays[:, 0:3].copy()).cuda().requires_grad_(True)
    d = torch.from_numpy(rays[:, 4:7].copy()).cuda().requires_grad_(True)
    t, u, v, prim = closest_hit_tuv(v0, v1, v2, o, d, bvh, tmax=100.0)
    hit = prim >= 0
    assert hit.sum() > 500
    target = torch.where(hit, t.detach() * 0.97, torch.zeros_like(t))
    loss = torch.where(hit, (t - target) ** 2, torch.zeros_like(t)).sum()
    loss.backward()
    g = [x.grad.detach().cpu().numpy().astype(np.float64) for x in (v0, v1, v2)]
    # FP64 oracle: the loss as a function of one vertex coordinate, hit ids held fixed
    prim_np = prim.cpu().numpy()
    tgt = target.cpu().numpy().astype(np.float64)
    R = rays.astype(np.float64)
    T = tris.astype(np.float64)

    def loss64(Tm, Rm=R):
        sel = prim_np >= 0
        a, b, c = Tm[prim_np[sel], 0], Tm[prim_np[sel], 1], Tm[prim_np[sel], 2]
        oo, dd = Rm[sel, 0:3], Rm[sel, 4:7]
        e1, e2, s = b - a, c - a, oo - a
        p = np.cross(dd, e2)
        det = (e1 * p).sum(1)
        q = np.cross(s, e1)
        tt = (e2 * q).sum(1) / det
        return ((tt - tgt[sel]) ** 2).sum()

    rng = np.random.default_rng(0)
    hit_tris = np.unique(prim_np[prim_np >= 0])
    errs = []
    for _ in range(1000):
        tri = int(rng.choice(hit_tris))
        k = int(rng.integers(0, 3))
        a = int(rng.integers(0, 3))
        h = 1e-4
        Tp = T.copy()
        Tp[tri, k, a] += h
        Tm = T.copy()
        Tm[tri, k, a] -= h
        fd = (loss64(Tp) - loss64(Tm)) / (2 * h)
        ad = g[k][tri, a]
        errs.append(abs(ad - fd) / max(abs(fd), 1e-3))
    errs = np.array(errs)
    assert np.median(errs) < 1e-3 and np.quantile(errs, 0.95) < 2e-2, (np.median(errs), np.quantile(errs, 0.95))
    # ray origins and directions against the same FP64 central differences
    go = o.grad.detach().cpu().numpy().astype(np.float64)
    gd = d.grad.detach().cpu().numpy().astype(np.float64)
    rerr = []
    for ray in rng.choice(np.nonzero(prim_np >= 0)[0], 100, replace=False):
        for col, grad in ((0, go), (4, gd)):
            a = int(rng.integers(0, 3))
            Rp, Rm = R.copy(), R.copy()
            Rp[ray, col + a] += 1e-4
            Rm[ray, col + a] -= 1e-4
            fd = (loss64(T, Rp) - loss64(T, Rm)) / 2e-4
            rerr.append(abs(grad[ray, a] - fd) / max(abs(fd), 1e-3))
    rerr = np.array(rerr)
    assert np.median(rerr) < 1e-3 and np.quantile(rerr, 0.95) < 2e-2, (np.median(rerr), np.quantile(rerr, 0.95))


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
    assert '"key": "morton30/aabb/binary/L4/b' in open(cache).read()
