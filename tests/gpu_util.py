"""Shared helpers of the GPU tests (all computation goes through libdipl_bvh.so)."""
import numpy as np
import torch

from diplodocus_b200 import accel as A


def build(tris, kind=A.AccelerationStructureType.kPloc, **kw):
    cfg = A.AccelerationStructureConfig(kind, **kw)
    bvh = A.GpuPlocBvh()
    bvh.Build(cfg, A.Stats(), torch.from_numpy(np.ascontiguousarray(tris, np.float32)))
    return bvh


def trace(bvh, rays, **kw):
    h = bvh.Intersect(A.Stats(), torch.from_numpy(np.ascontiguousarray(rays, np.float32)), **kw)
    torch.cuda.synchronize()
    bvh.check_errors()
    return (h.prim.cpu().numpy(), h.t.cpu().numpy(), h.u.cpu().numpy(), h.v.cpu().numpy())


def fbits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)
