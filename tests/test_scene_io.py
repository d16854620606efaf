"""OBJ scene path and statistics export.

CPU: the library's host-side loader (dipl_obj_scene_load, through diplodocus_b200/scene_io.py) against the reference ObjSceneLoader's output on the
hand-written fixture scene (golden vectors from tests/golden/make_obj_golden.py) and, where the reference
harness is built, against the reference loader directly (fixtures, and the reference's own Cornell scenes when
its tree is present); the console statistics text against the reference ConsoleStatsExporter; the CSV exporter.
GPU: a loaded scene built and traced on the device, every primary and bounce hit equal to brute force, and the
frame's statistics.
"""
import io
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN, bits, load_golden
from diplodocus_b200 import accel as A
from diplodocus_b200 import scene_io as SI
from diplodocus_b200 import stats_io as SIO

OBJ_DIR = os.path.join(GOLDEN, "obj")


def scene_arrays(sc):
    mv = np.array([np.concatenate([m.ambient, m.diffuse, m.specular, m.transmittance, m.emission,
                                   [m.shininess, m.ior, m.r_ior, m.dissolve]]) for m in sc.materials],
                  np.float32).reshape(-1, 19)
    return {
        "positions": sc.positions, "normals": sc.normals, "geom_normals": sc.geom_normals,
        "material_ids": sc.material_ids, "has_vertex_normals": sc.has_vertex_normals, "material_values": mv,
        "material_names": [m.name for m in sc.materials],
        "area_light_triangles": np.array([a.triangle_id for a in sc.area_lights], np.int32),
        "area_light_colors": np.array([a.color for a in sc.area_lights], np.float32).reshape(-1, 3),
        "area_light_areas": np.array([a.surface_area for a in sc.area_lights], np.float32),
        "camera": np.concatenate([sc.camera.pos, sc.camera.dir, sc.camera.up, [sc.camera.fov, sc.camera.far]])
        .astype(np.float32),
        "point_lights": np.array([np.concatenate([p.pos, p.color, [p.power]]) for p in sc.point_lights],
                                 np.float32).reshape(-1, 7),
    }


def assert_same_scene(mine, ref):
    assert len(mine["positions"]) == len(ref["positions"])
    for k in ("positions", "normals", "geom_normals", "material_values", "area_light_colors", "area_light_areas",
              "camera", "point_lights"):
        np.testing.assert_array_equal(bits(mine[k]), bits(ref[k]), err_msg=k)
    for k in ("material_ids", "has_vertex_normals", "area_light_triangles"):
        np.testing.assert_array_equal(mine[k], np.asarray(ref[k]), err_msg=k)
    assert list(mine["material_names"]) == [str(x) for x in ref["material_names"]]


def test_fixture_scene_equals_reference_loader_golden():
    sc = SI.load_obj_scene(OBJ_DIR, "room")
    assert sc is not None
    assert_same_scene(scene_arrays(sc), load_golden("obj_room"))
    # what the fixture exercises: quads on both diagonals, a convex pentagon, concave hexagon and heptagon,
    # faces without material (-1), duplicate material names across two MTL files, an emissive pentagon
    assert len(sc) == 24
    assert (sc.material_ids == -1).sum() == 2
    assert [a.triangle_id for a in sc.area_lights] == [12, 13, 14]
    assert sc.has_vertex_normals.sum() == 8


def test_failures_return_none_like_the_reference():
    assert SI.load_obj_scene(OBJ_DIR, "broken_meta") is None   # unknown metadata token
    assert SI.load_obj_scene(OBJ_DIR, "missing_obj") is None   # no .obj beside the .meta
    assert SI.load_obj_scene(OBJ_DIR, "no_such_scene") is None  # no .meta


@pytest.mark.parametrize("name", ["room", "broken_meta", "missing_obj"])
def test_fixtures_equal_reference_loader(ref, name):
    mine, theirs = SI.load_obj_scene(OBJ_DIR, name), ref.obj_scene(OBJ_DIR, name)
    assert (mine is None) == (theirs is None)
    if mine is not None:
        assert_same_scene(scene_arrays(mine), theirs)


@pytest.mark.parametrize("name", ["CornellBox-Original", "CornellBox-Sphere"])
def test_reference_cornell_scenes_equal_reference_loader(ref, name):
    import oracle as O
    res = os.path.join(O.REFERENCE_TREE, "res")
    if not os.path.exists(os.path.join(res, name + ".obj")):
        pytest.skip("the reference's scene files are not here")
    assert_same_scene(scene_arrays(SI.load_obj_scene(res, name)), ref.obj_scene(res, name))


def write_scene(tmp_path, name, obj, meta="cam_pos 0 0 0\n", mtl=None):
    (tmp_path / f"{name}.meta").write_text(meta)
    (tmp_path / f"{name}.obj").write_text(obj)
    if mtl is not None:
        (tmp_path / f"{name}.mtl").write_text(mtl)
    return str(tmp_path)


def test_number_tokens_read_like_tinyobj(tmp_path):
    # the longest decimal prefix of a token (the reference's CornellBox-Sphere.obj has "-0.2200."), nan / inf
    d = write_scene(tmp_path, "nums", "v 1e -0.2200. .5\nv -inf 2 3\nv 0 0 0\nf 1 2 3\n")
    sc = SI.load_obj_scene(d, "nums")
    p = sc.positions[0]
    assert p[0] == np.float32(1.0) and p[1] == np.float32(-0.22) and p[2] == np.float32(0.5)
    assert np.isneginf(p[3])
    assert SI.load_obj_scene(write_scene(tmp_path, "bad", "v abc 0 0\nv 0 0 0\nv 1 1 1\nf 1 2 3\n"), "bad") is None
    assert SI.load_obj_scene(write_scene(tmp_path, "big", "v 1e400 0 0\nv 0 0 0\nv 1 1 1\nf 1 2 3\n"), "big") is None
    assert SI.load_obj_scene(write_scene(tmp_path, "zero", "v 0 0 0\nv 1 0 0\nv 1 1 1\nf 0 1 2\n"), "zero") is None
    assert SI.load_obj_scene(write_scene(tmp_path, "oob", "v 0 0 0\nv 1 0 0\nf 1 2 9\n"), "oob") is None
    assert SI.load_obj_scene(write_scene(tmp_path, "m", "v 0 0 0\nv 1 0 0\nv 1 1 0\nf 1 2 3\n",
                                         meta="cam_fov 0.5x\n"), "m") is None
    import oracle as O
    if os.path.exists(O.REF_LIB):
        r = O.RefOracle()
        assert_same_scene(scene_arrays(sc), r.obj_scene(d, "nums"))
        for name in ("bad", "big", "zero"):
            assert r.obj_scene(str(tmp_path), name) is None


def test_quad_split_takes_the_shorter_diagonal(tmp_path):
    obj = ("v 0 0 0\nv 4 0 0\nv 4 1 0\nv 0 1 0\nf 1 2 3 4\n"   # diagonals equal: 0-1-3 / 1-2-3
           "v 0 0 1\nv 1 0 1\nv 3 3 1\nv 0 1 1\nf 5 6 7 8\n"   # 6-8 is the short one
           "v 0 0 2\nv 3 0 2\nv 1 1 2\nv 0 3 2\nf 9 10 11 12\n")  # 9-11 is the short one
    sc = SI.load_obj_scene(write_scene(tmp_path, "q", obj), "q")
    tri = sc.triangles()
    assert len(sc) == 6
    np.testing.assert_array_equal(tri[2], [[0, 0, 1], [1, 0, 1], [0, 1, 1]])
    np.testing.assert_array_equal(tri[3], [[1, 0, 1], [3, 3, 1], [0, 1, 1]])
    np.testing.assert_array_equal(tri[4], [[0, 0, 2], [3, 0, 2], [1, 1, 2]])
    np.testing.assert_array_equal(tri[5], [[0, 0, 2], [1, 1, 2], [0, 3, 2]])


def test_large_file_parsed_in_chunks_equals_file_order(tmp_path):
    """A file large enough to be parsed in several chunks: relative indices that reach across chunk boundaries,
    material switches, groups and quads; the triangles, their order and material ids are known by
    construction (and equal the reference loader's where its harness is built)."""
    rng = np.random.default_rng(5)
    n = 150_000
    tri = rng.uniform(-10, 10, size=(n, 3, 3)).astype(np.float32)
    lines = ["mtllib m.mtl"]
    want_pos, want_mat = [], []
    mat = -1
    for i in range(n):
        if i % 997 == 0:
            mat = (i // 997) % 3
            lines.append(f"usemtl m{mat}")
        if i % 4999 == 0:
            lines.append(f"g group{i}")
        for k in range(3):
            lines.append("v %.9g %.9g %.9g" % tuple(tri[i, k]))
        if i % 7 == 3 and i > 0:
            # a quad over the previous triangle's v2 and this one's: split along the shorter diagonal
            lines.append("f -4 -3 -2 -1")
            q = np.concatenate([tri[i - 1, 2:3], tri[i]])
            d02, d13 = q[2] - q[0], q[3] - q[1]
            s02 = np.float32(np.float32(d02[0] * d02[0] + d02[1] * d02[1]) + d02[2] * d02[2])
            s13 = np.float32(np.float32(d13[0] * d13[0] + d13[1] * d13[1]) + d13[2] * d13[2])
            for t in ([(0, 1, 2), (0, 2, 3)] if s02 < s13 else [(0, 1, 3), (1, 2, 3)]):
                want_pos.append(q[list(t)])
                want_mat.append(mat)
        else:
            lines.append(f"f {3 * i + 1 if i % 2 else -3} {3 * i + 2 if i % 2 else -2} -1")
            want_pos.append(tri[i])
            want_mat.append(mat)
    (tmp_path / "big.obj").write_text("\n".join(lines) + "\n")
    (tmp_path / "big.meta").write_text("cam_pos 0 0 0\n")
    (tmp_path / "m.mtl").write_text("newmtl m0\nKd 1 0 0\nnewmtl m1\nKd 0 1 0\nnewmtl m2\nKe 1 1 1\n")
    assert (tmp_path / "big.obj").stat().st_size > 16 << 20
    sc = SI.load_obj_scene(str(tmp_path), "big")
    np.testing.assert_array_equal(bits(sc.positions), bits(np.array(want_pos).reshape(-1, 9)))
    np.testing.assert_array_equal(sc.material_ids, np.array(want_mat, np.int32))
    assert [a.triangle_id for a in sc.area_lights] == list(np.nonzero(np.array(want_mat) == 2)[0])
    import oracle as O
    if os.path.exists(O.REF_LIB):
        assert_same_scene(scene_arrays(sc), O.RefOracle().obj_scene(str(tmp_path), "big"))


def test_loader_needs_no_device_and_checks_arguments():
    import ctypes as C
    from diplodocus_b200 import _lib as L
    lib = L.load()
    h = C.c_void_p(0)
    assert lib.dipl_obj_scene_load(None, b"x", C.byref(h)) == 1
    assert lib.dipl_obj_scene_load(OBJ_DIR.encode(), b"no_such_scene", C.byref(h)) == L.DIPL_ERR_IO
    assert b"cannot read" in lib.dipl_last_error()
    assert lib.dipl_status_string(L.DIPL_ERR_IO) == b"DIPL_ERR_IO"


def test_stats_console_text_equals_reference(ref):
    cases = [([1.23456, 262144, 100000, 0], [12.5, 1999, 999, 1000, 123456, 362144, 54321, 98765]),
             ([0, 0, 0, 0], [0, 0, 0, 0, 0, 0, 0, 0]),
             ([0.000123, 1, 2, 3], [1234.5678, 1, 2, 3, 999, 7, 3, 0])]
    for rt, ac in cases:
        s = A.Stats(A.RaytracingStats(rt[0], *map(int, rt[1:])), A.AccelerationStats(ac[0], *map(int, ac[1:])))
        mine = SIO.ConsoleStatsExporter().text(s).splitlines()
        theirs = ref.console_stats(rt, ac).splitlines()
        assert len(mine) == len(theirs)
        for a, b in zip(mine, theirs):
            if a.startswith(" Traversals per query:"):
                # the reference divides the intersection count here; this divides the traversal count
                q, tcount = int(ac[5]), int(ac[7])
                want = 0.0 if q == 0 or tcount == 0 else float(np.float32(tcount) / np.float32(q))
                assert a.split(":")[1].strip() == format(want, ".3g")
            else:
                assert a == b


def test_stats_csv_round_trip(tmp_path):
    s1 = A.Stats(A.RaytracingStats(0.5, 10, 4, 0), A.AccelerationStats(1.5, 7, 3, 4, 1024, 14, 9, 33))
    s2 = A.Stats(A.RaytracingStats(2.0, 1 << 40, 3, 1), A.AccelerationStats(0.25, 1, 0, 1, 64, 5, 1 << 35, 7))
    cfg = SIO.StatsExportConfig(SIO.parse_stats_export_format("csv"), path=str(tmp_path / "stats.csv"))
    exp = SIO.CreateStatsExporter(cfg)
    assert isinstance(exp, SIO.CsvStatsExporter)
    exp.ExportOne(cfg, s1)
    exp.ExportOne(cfg, s2)  # appends without a second header
    text = (tmp_path / "stats.csv").read_text()
    assert text.splitlines()[0] == ",".join(SIO.CSV_COLUMNS) and text.count("raytracing_time") == 1
    assert SIO.read_stats_csv(str(tmp_path / "stats.csv")) == [s1, s2]  # 64-bit counts survive
    buf = io.StringIO()
    SIO.CsvStatsExporter(buf).ExportAll(cfg, [s1])
    assert SIO.read_stats_csv(buf.getvalue()) == [s1]
    with pytest.raises(ValueError):
        SIO.parse_stats_export_format("json")
    assert isinstance(SIO.CreateStatsExporter(SIO.StatsExportConfig()), SIO.ConsoleStatsExporter)


@pytest.mark.gpu
def test_obj_scene_frame_hits_equal_brute_force(orc):
    """file -> device SoA -> PLOC build -> generate -> trace -> bounce -> trace; both hit sets equal brute
    force on the loaded triangles, and the frame's statistics are filled."""
    sc = SI.load_obj_scene(OBJ_DIR, "room")
    stats = A.Stats()
    bvh, (rays, hits, bounce, bhits) = SI.render_scene_frame(sc, 80, 60, seed=7, stats=stats)
    tris = sc.triangles()
    for r, h in ((rays, hits), (bounce, bhits)):
        want = orc.brute(tris, r.cpu().numpy())
        np.testing.assert_array_equal(h.prim.cpu().numpy(), want.prim)
        np.testing.assert_array_equal(bits(h.t.cpu().numpy()), bits(want.t))
    n_hits = int((hits.prim >= 0).sum().item())
    assert n_hits > 1000
    assert stats.rt_stats.primary_ray_count == 80 * 60
    assert stats.rt_stats.secondary_ray_count == n_hits
    assert stats.rt_stats.raytracing_time > 0.0
    assert stats.accel_stats.inner_node_count > 0 and stats.accel_stats.query_count == 2 * 80 * 60
    text = SIO.ConsoleStatsExporter().text(stats)
    assert f" Primary ray count:             {80 * 60}" in text
