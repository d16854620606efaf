"""The reference-side adapter (diplodocus_b200/adapter/gpu_ploc_bvh.h): GpuPlocBvh implementing the reference's
AccelerationStructure, compiled against the reference's own headers with g++ (C++20) and driven like the
reference's renderer drives an acceleration structure."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from conftest import load_golden


def test_adapter_compiles_against_the_reference_headers():
    """g++ -std=c++20 -Wall on the adapter + driver with the reference's src/ on the include path (CPU only)."""
    if not os.path.isdir(O.REFERENCE_TREE):
        pytest.skip("the reference tree is not here (the adapter is compiled where it is)")
    lib = os.path.join(os.path.dirname(O.HERE), "diplodocus_b200", "lib", "libdipl_bvh.so")
    if not os.path.exists(lib):
        pytest.skip("libdipl_bvh.so is not built")
    r = subprocess.run(["make", "-C", O.HERE, "-B", "adapter"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "warning" not in r.stderr
    assert os.access(O.ADAPTER_CHECK, os.X_OK)


def _run(tmp_path, kind, tris, rays, per_ray):
    tp, rp, op = tmp_path / "t.bin", tmp_path / "r.bin", tmp_path / "o.bin"
    np.ascontiguousarray(tris, np.float32).tofile(tp)
    np.ascontiguousarray(rays, np.float32).tofile(rp)
    r = subprocess.run([O.ADAPTER_CHECK, kind, str(tp), str(rp), str(op), str(per_ray)], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    raw = np.fromfile(op, np.uint8)
    k = int(raw[:4].view(np.int32)[0])
    nr = len(rays)
    off = 4
    batch = raw[off: off + 16 * nr].view(np.int32).reshape(nr, 4)
    off += 16 * nr
    one = raw[off: off + 16 * k].view(np.int32).reshape(k, 4)
    off += 16 * k
    occ_b = raw[off: off + nr].astype(bool)
    off += nr
    occ_1 = raw[off: off + k].astype(bool)
    off += k
    counters = raw[off: off + 8].view(np.int32)
    return batch, one, occ_b, occ_1, counters


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["ploc", "ploc_emc", "ploc_sobb", "ploc_emc_sobb"])
@pytest.mark.parametrize("name", ["small_scene", "soup_2k", "duplicates_ties"])
def test_adapter_answers_equal_the_reference_brute_force(orc, tmp_path, kind, name):
    """GpuPlocBvh::Build, then Intersect / IntersectAny one ray at a time (the CPU renderer's calls) and the batch
    paths: hit ids, t, b1 and b2 bit-equal to DummyAccelerationStucture::Intersect's, occlusion equal to the any-hit
    brute force (tmin < t < tmax)."""
    if not os.access(O.ADAPTER_CHECK, os.X_OK):
        pytest.skip("the adapter driver is built where the reference tree is (oracle/Makefile, target adapter)")
    g = load_golden(name)
    batch, one, occ_b, occ_1, counters = _run(tmp_path, kind, g["tris"], g["rays"], 300)
    want = np.stack([g["brute_prim"], g["brute_t"].view(np.int32), g["brute_u"].view(np.int32),
                     g["brute_v"].view(np.int32)], 1)
    want[g["brute_prim"] < 0, 1:] = np.array([np.inf, 0, 0], np.float32).view(np.int32)
    np.testing.assert_array_equal(batch, want)
    np.testing.assert_array_equal(one, want[: len(one)])
    any_ref = orc.brute_any(g["tris"], g["rays"])
    np.testing.assert_array_equal(occ_b, any_ref)
    np.testing.assert_array_equal(occ_1, any_ref[: len(occ_1)])
    assert counters[0] == 2 * len(g["rays"]) + 2 * len(one)  # query_count: every traced ray, batch and one by one
