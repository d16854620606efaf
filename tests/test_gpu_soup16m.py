"""GPU: the 16M-triangle soup at full size (16,777,216 triangles, 16,777,216 random rays).

Every layout the engine traces is checked on the same sample of rays against the reference's own brute force
(DummyAccelerationStucture::Intersect, compiled from its sources; lowest-id tie rule) and SBvh, and every hit
of the full batch re-tests to the same bits under the reference's Moller-Trumbore arithmetic."""
import numpy as np
import pytest
import torch

import oracle as O
from diplodocus_b200 import accel as A
from diplodocus_b200 import scenes as S
from gpu_util import build

pytestmark = pytest.mark.gpu

N = 16 * 1024 * 1024
SAMPLE = 4096
FORMS = [("ploc_emc", A.AccelerationStructureType.kPlocEmc, "binary"),
         ("ploc_emc_split40", A.AccelerationStructureType.kPlocEmc, "binary"),
         ("ploc", A.AccelerationStructureType.kPloc, "binary"),
         ("ploc_emc_sobb", A.AccelerationStructureType.kPlocEmcSobb, "binary"),
         ("ploc_emc_wide8_q8", A.AccelerationStructureType.kPlocEmc, "wide8_q8")]


@pytest.fixture(scope="module")
def soup_and_answers(ref):
    tris = S.soup(N, seed=3)
    rays = S.random_rays(N, seed=3)
    idx = np.linspace(0, N - 1, SAMPLE).astype(np.int64)
    sample = np.ascontiguousarray(rays[idx])
    brute = ref.brute(tris, sample, chunk=8192)
    sb = ref.sbvh(tris)
    sbvh = sb.trace(sample)
    sb.close()
    return tris, rays, idx, brute, sbvh


def _hits(bvh, rays_dev):
    h = bvh.Intersect(A.Stats(), rays_dev)
    torch.cuda.synchronize()
    bvh.check_errors()
    return h.prim.cpu().numpy(), h.t.cpu().numpy(), h.u.cpu().numpy(), h.v.cpu().numpy()


def test_soup16m_forms_bit_exact_on_a_ray_sample_and_every_hit_retests(orc, soup_and_answers):
    tris, rays, idx, brute, sbvh = soup_and_answers
    rays_dev = torch.from_numpy(rays).cuda()
    first = None
    for name, kind, layout in FORMS:
        bvh = build(tris, kind, layout=layout, split_budget=40 if name.endswith("split40") else 0)
        prim, t, u, v = _hits(bvh, rays_dev)
        cls = O.classify_hits(prim[idx], t[idx], u[idx], v[idx], brute, sbvh)
        assert cls["E"] == SAMPLE and cls["F"] == 0 and cls["T"] == 0, (name, cls)
        assert cls["vs_sbvh"]["F"] == 0, (name, cls)
        if first is None:
            first = prim
            # the full batch: each reported hit is the reference arithmetic's answer for that ray and triangle
            hit = prim >= 0
            h = orc.test_pairs(tris, rays[hit], prim[hit])
            np.testing.assert_array_equal(h.t.view(np.uint32), t[hit].view(np.uint32))
            np.testing.assert_array_equal(h.u.view(np.uint32), u[hit].view(np.uint32))
            np.testing.assert_array_equal(h.v.view(np.uint32), v[hit].view(np.uint32))
        else:
            # every form finds the same closest hit for every one of the 16M rays
            np.testing.assert_array_equal(prim, first)
        bvh.close()
        del bvh
        torch.cuda.empty_cache()
