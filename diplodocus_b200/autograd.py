"""Differentiation form: closest-hit t/u/v as a torch.autograd.Function over the engine's C ABI.

Forward: build (once, outside) + dipl_bvh_trace_closest; the hit ids are discrete and held fixed.
Backward: dipl_trace_adjoint, the hand-written adjoint of (t, u, v) with respect to the triangle vertices
and the ray origins and directions. This wrapper exists for checking the adjoint against finite
differences and for gradient-based callers; all computation is in libdipl_bvh.so.
"""
from __future__ import annotations

import torch

from . import accel as A


class ClosestHitTUV(torch.autograd.Function):
    """(v0, v1, v2, origins, directions) -> (t, u, v) of the closest hit of every ray (misses: inf, 0, 0).

    ``bvh`` is a GpuPlocBvh built over the same vertices; ``rays`` carries tmin/tmax. Vertex tensors are the
    SoA float3 arrays (N, 3); origins/directions are (R, 3) float32 on the GPU.
    """

    @staticmethod
    def forward(ctx, v0, v1, v2, origins, directions, bvh, tmin, tmax, leaf_test="ref_mt"):
        rays = torch.empty((origins.shape[0], 8), dtype=torch.float32, device=origins.device)
        rays[:, 0:3] = origins
        rays[:, 3] = tmin
        rays[:, 4:7] = directions
        rays[:, 7] = tmax
        hits = bvh.Intersect(A.Stats(), rays, leaf_test=leaf_test)
        ctx.save_for_backward(v0.detach().contiguous(), v1.detach().contiguous(), v2.detach().contiguous(), rays,
                              hits.raw)
        ctx.mark_non_differentiable(hits.prim)
        return hits.t.clone(), hits.u.clone(), hits.v.clone(), hits.prim.clone()

    @staticmethod
    def backward(ctx, gt, gu, gv, _gprim):
        v0, v1, v2, rays, raw = ctx.saved_tensors
        f = raw.view(torch.float32)
        hits = A.Hits(raw[:, 0], f[:, 1], f[:, 2], f[:, 3], raw)
        dtuv = torch.stack([torch.nan_to_num(g, nan=0.0, posinf=0.0, neginf=0.0) if g is not None
                            else torch.zeros_like(hits.t) for g in (gt, gu, gv)], dim=1)
        dv0, dv1, dv2, dorig, ddir = A.trace_adjoint((v0, v1, v2), rays, hits, dtuv)
        return dv0, dv1, dv2, dorig, ddir, None, None, None, None


def closest_hit_tuv(v0, v1, v2, origins, directions, bvh, tmin=1e-6, tmax=3.4028234663852886e38, leaf_test="ref_mt"):
    return ClosestHitTUV.apply(v0, v1, v2, origins, directions, bvh, tmin, tmax, leaf_test)
