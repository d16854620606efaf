"""Generates the golden fixtures of tests/golden/ from the REFERENCE's own code.

Run in a tree where the reference is present (it builds oracle/_ref/libref_oracle.so from the reference's
sources): ``python tests/golden/make_golden.py``. Each fixture holds seeded triangles and rays and the
reference's answers on them:

* brute_*: DummyAccelerationStucture::Intersect (src/acceleration/dummy_acceleration_structure.cc:21-64),
  the lowest-id closest hit, with Triangle::IntersectRay (src/scene/triangle.cc:10-43);
* sbvh_*:  SBvh::Build + SBvh::Intersect (src/acceleration/sbvh.cc:17-145), defaults
  (bin_count 16, max_triangles_per_leaf 4, max_depth 32), and its FP64 SAH cost.
t, u, v are stored as float32 so the bit patterns are the reference's.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402
from diplodocus_b200 import scenes as S  # noqa: E402


def cases():
    # small scene (box + sphere) at reduced resolution, primary + bounce rays
    tris, rays = S.small_scene(seed=1, width=96, height=96, sphere_nu=32, sphere_nv=16)
    yield "small_scene", tris, rays, True
    # the full small-scene mesh (10 + 3968 triangles), a 64x64 pinhole subset
    tris, rays = S.small_scene(seed=7, width=64, height=64)
    yield "small_scene_full_mesh", tris, rays, True
    # displaced sphere, small
    tris = S.uv_sphere(64, 32, 1.0, (0, 0, 0), displacement=0.05, seed=2)
    yield "displaced_sphere_64x32", tris, S.sphere_inward_rays(4096, seed=2), False
    # soup, small (heavy-tailed sizes, 29% tiny determinants)
    yield "soup_2k", S.soup(2000, seed=3), S.random_rays(4096, seed=3), False
    # degenerate: duplicate triangles and exact-t ties
    base = S.open_box()
    dup = np.concatenate([base, base, base[::-1]])
    o = S.pinhole_rays(32, 32, **S.SMALL_CAMERA)
    yield "duplicates_ties", dup, o, False


def main():
    O.build()
    ref = O.RefOracle()
    for name, tris, rays, bounce in cases():
        tris = np.ascontiguousarray(tris, np.float32)
        rays = np.ascontiguousarray(rays, np.float32)
        if bounce:
            h0 = ref.brute(tris, rays)
            br, mask = S.bounce_rays(tris, rays, h0.prim, h0.t, seed=11)
            rays = np.concatenate([rays, br[mask]])
        hb = ref.brute(tris, rays)
        sb = ref.sbvh(tris)
        hs = sb.trace(rays)
        sah, ni, nl = sb.sah_cost()
        out = os.path.join(HERE, name + ".npz")
        np.savez_compressed(out, tris=tris, rays=rays, brute_prim=hb.prim, brute_t=hb.t, brute_u=hb.u,
                            brute_v=hb.v, sbvh_prim=hs.prim, sbvh_t=hs.t, sbvh_u=hs.u, sbvh_v=hs.v,
                            sbvh_sah=np.float64(sah), sbvh_inner=np.int64(ni), sbvh_leaves=np.int64(nl))
        agree = float((hb.prim == hs.prim).mean())
        print(f"{name}: {len(tris)} tris, {len(rays)} rays, hits {(hb.prim >= 0).sum()}, "
              f"sbvh agrees {agree:.4f}, sbvh sah {sah:.3f} -> {os.path.basename(out)} "
              f"({os.path.getsize(out) // 1024} KiB)")


if __name__ == "__main__":
    main()
