"""TEST INFRASTRUCTURE — CHECKER ONLY.

ctypes bindings for the two oracles:

* ``RefOracle``  — the reference's own SBvh / brute force / Moller-Trumbore / OBJ scene loader / console
  statistics exporter compiled from its
  sources (oracle/_ref/libref_oracle.so, built by oracle/Makefile in a tree where the reference
  is present; the built file then travels with the repository snapshot).
* ``Oracle``     — the plain-C restatement in oracle/dipl_oracle.c (oracle/libdipl_oracle.so).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libref_oracle.so")
ADAPTER_CHECK = os.path.join(HERE, "_ref", "adapter_check")
ORC_LIB = os.path.join(HERE, "libdipl_oracle.so")
# where the reference tree is compiled from (the reference harness is built only where it exists)
REFERENCE_TREE = os.environ.get("DIPL_REFERENCE_TREE", "/root/reference")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")


def build(force=False):
    """Compile the C restatement always, and the reference harness when the reference tree is here."""
    targets = ["libdipl_oracle.so"]
    if os.path.isdir(REFERENCE_TREE):
        targets += ["ref", "adapter"]
    cmd = ["make", "-C", HERE] + (["-B"] if force else []) + targets
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)


def _tris(t):
    t = np.ascontiguousarray(t, dtype=np.float32)
    assert t.ndim == 3 and t.shape[1:] == (3, 3), t.shape
    return t


def _rays(r):
    r = np.ascontiguousarray(r, dtype=np.float32)
    assert r.ndim == 2 and r.shape[1] == 8, r.shape
    return r


class Hits:
    """Closest-hit records: prim (int32, -1 = miss), t, u (= b1), v (= b2)."""

    def __init__(self, n):
        self.prim = np.empty(n, np.int32)
        self.t = np.empty(n, np.float32)
        self.u = np.empty(n, np.float32)
        self.v = np.empty(n, np.float32)


class RefOracle:
    """The reference's own code (SBvh, DummyAccelerationStucture, Triangle::IntersectRay)."""

    def __init__(self, path=REF_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (run make -C oracle ref where the reference tree exists)")
        L = self.lib = C.CDLL(path)
        L.ref_sbvh_build.restype = C.c_void_p
        L.ref_sbvh_build.argtypes = [_f32p, C.c_int64, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double)]
        L.ref_sbvh_rebuild.restype = C.c_double
        L.ref_sbvh_rebuild.argtypes = [C.c_void_p]
        L.ref_sbvh_destroy.argtypes = [C.c_void_p]
        L.ref_sbvh_trace.argtypes = [C.c_void_p, _f32p, C.c_int64, _i32p, _f32p, _f32p, _f32p, C.c_int, C.c_int,
                                     _i64p]
        L.ref_sbvh_sah_cost.restype = C.c_double
        L.ref_sbvh_sah_cost.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        L.ref_brute_trace.argtypes = [_f32p, C.c_int64, _f32p, C.c_int64, _i32p, _f32p, _f32p, _f32p, C.c_int,
                                      C.c_int]
        L.ref_brute_trace_chunked.argtypes = [_f32p, C.c_int64, _f32p, C.c_int64, _i32p, _f32p, _f32p, _f32p,
                                              C.c_int, C.c_int, C.c_int64]
        L.ref_intersect_one.restype = C.c_float
        L.ref_intersect_one.argtypes = [_f32p, _f32p, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.ref_obj_scene_load.restype = C.c_void_p
        L.ref_obj_scene_load.argtypes = [C.c_char_p, C.c_char_p]
        L.ref_obj_scene_free.argtypes = [C.c_void_p]
        L.ref_obj_scene_counts.argtypes = [C.c_void_p, _i64p]
        L.ref_obj_scene_triangles.argtypes = [C.c_void_p, _f32p, _f32p, _f32p, _i32p, C.c_void_p]
        L.ref_obj_scene_materials.argtypes = [C.c_void_p, _f32p, C.c_void_p]
        L.ref_obj_scene_area_lights.argtypes = [C.c_void_p, _i32p, _f32p, _f32p]
        L.ref_obj_scene_camera_lights.argtypes = [C.c_void_p, _f32p, _f32p]
        L.ref_console_stats.argtypes = [_f64p, _f64p]

    def sbvh(self, tris, max_depth=32, max_triangles_per_leaf=4, bin_count=16):
        return SBvh(self, _tris(tris), max_depth, max_triangles_per_leaf, bin_count)

    def obj_scene(self, dirpath, name):
        """The reference ObjSceneLoader::Load (obj_scene_loader.cc:189-205) on <dirpath>/<name>.{meta,obj}: a dict
        of numpy arrays, or None where the reference loader fails."""
        L = self.lib
        h = L.ref_obj_scene_load(str(dirpath).encode(), str(name).encode())
        if not h:
            return None
        try:
            cnt = np.zeros(4, np.int64)
            L.ref_obj_scene_counts(h, cnt)
            nt, nm, na, npl = (int(x) for x in cnt)
            pos = np.zeros((nt, 9), np.float32)
            nrm = np.zeros((nt, 9), np.float32)
            geom = np.zeros((nt, 3), np.float32)
            mat = np.zeros(nt, np.int32)
            has_n = np.zeros(nt, np.uint8)
            L.ref_obj_scene_triangles(h, pos, nrm, geom, mat, has_n.ctypes.data_as(C.c_void_p))
            mvals = np.zeros((nm, 19), np.float32)
            names = np.zeros((nm, 64), np.uint8)
            L.ref_obj_scene_materials(h, mvals, names.ctypes.data_as(C.c_void_p))
            al_id = np.zeros(na, np.int32)
            al_color = np.zeros((na, 3), np.float32)
            al_area = np.zeros(na, np.float32)
            L.ref_obj_scene_area_lights(h, al_id, al_color, al_area)
            cam = np.zeros(11, np.float32)
            lights = np.zeros((npl, 7), np.float32)
            L.ref_obj_scene_camera_lights(h, cam, lights)
        finally:
            L.ref_obj_scene_free(h)
        return {"positions": pos, "normals": nrm, "geom_normals": geom, "material_ids": mat,
                "has_vertex_normals": has_n.astype(bool), "material_values": mvals,
                "material_names": [bytes(r).split(b"\0", 1)[0].decode() for r in names],
                "area_light_triangles": al_id, "area_light_colors": al_color, "area_light_areas": al_area,
                "camera": cam, "point_lights": lights}

    def console_stats(self, rt, accel):
        """The reference ConsoleStatsExporter's text for the given values (rt: 4, accel: 8 numbers, the order of
        RaytracingStats / AccelerationStats), captured from the process's stdout."""
        import sys
        import tempfile
        sys.stdout.flush()
        with tempfile.TemporaryFile() as tmp:
            saved = os.dup(1)
            try:
                os.dup2(tmp.fileno(), 1)
                self.lib.ref_console_stats(np.asarray(rt, np.float64), np.asarray(accel, np.float64))
            finally:
                os.dup2(saved, 1)
                os.close(saved)
            tmp.seek(0)
            return tmp.read().decode()

    def brute(self, tris, rays, backface=False, threads=None, chunk=None):
        """DummyAccelerationStucture::Intersect on every ray. With ``chunk``, the same comparisons run chunk by chunk
        of the triangles (ref_brute_trace_chunked: identical records, far fewer cache misses on large scenes)."""
        tris, rays = _tris(tris), _rays(rays)
        h = Hits(len(rays))
        nt = int(threads or os.cpu_count() or 1)
        if chunk:
            self.lib.ref_brute_trace_chunked(tris, len(tris), rays, len(rays), h.prim, h.t, h.u, h.v, int(backface),
                                             nt, int(chunk))
        else:
            self.lib.ref_brute_trace(tris, len(tris), rays, len(rays), h.prim, h.t, h.u, h.v, int(backface), nt)
        return h


class SBvh:
    def __init__(self, ref, tris, max_depth, max_leaf, bins):
        self.ref, self.tris = ref, tris
        ms = C.c_double(0.0)
        self.h = ref.lib.ref_sbvh_build(tris, len(tris), max_depth, max_leaf, bins, C.byref(ms))
        self.build_ms = ms.value

    def rebuild_ms(self):
        return self.ref.lib.ref_sbvh_rebuild(self.h)

    def trace(self, rays, backface=False, threads=None):
        rays = _rays(rays)
        h = Hits(len(rays))
        cnt = np.zeros(3, np.int64)
        self.ref.lib.ref_sbvh_trace(self.h, rays, len(rays), h.prim, h.t, h.u, h.v, int(backface),
                                    int(threads or os.cpu_count() or 1), cnt)
        h.counters = cnt
        return h

    def sah_cost(self):
        ni, nl = C.c_int64(0), C.c_int64(0)
        c = self.ref.lib.ref_sbvh_sah_cost(self.h, C.byref(ni), C.byref(nl))
        return c, ni.value, nl.value

    def close(self):
        if self.h:
            self.ref.lib.ref_sbvh_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Oracle:
    """The plain-C restatement (oracle/dipl_oracle.c)."""

    def __init__(self, path=ORC_LIB):
        if not os.path.exists(path):
            build()
        L = self.lib = C.CDLL(path)
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_mt.restype = C.c_float
        L.orc_mt.argtypes = [_f32p, _f32p, _f32p, _f32p, _f32p, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.orc_wt.restype = C.c_float
        L.orc_wt.argtypes = L.orc_mt.argtypes
        L.orc_brute_closest.argtypes = [_f32p, C.c_int64, _f32p, C.c_int64, C.c_int, C.c_int, _i32p, _f32p, _f32p,
                                        _f32p]
        L.orc_brute_any.argtypes = [_f32p, C.c_int64, _f32p, C.c_int64, C.c_int, C.c_int, _u8p]
        L.orc_intersect_f64.argtypes = [_f32p, _f32p, C.c_int64, _i32p, _f64p, _f64p, _f64p]
        L.orc_brute_closest_f64.argtypes = [_f32p, C.c_int64, _f32p, C.c_int64, _i32p, _f64p]
        L.orc_scene_bounds.argtypes = [_f32p, C.c_int64, _f32p, _f32p, _f32p, _f32p]
        L.orc_morton30.argtypes = [_f32p, C.c_int64, _f32p, _f32p, _u32p]
        L.orc_emc60_plan.argtypes = [_f32p, _f32p, C.c_float, _i32p, _u64p]
        L.orc_scene_diag.restype = C.c_float
        L.orc_scene_diag.argtypes = [_f32p, _f32p]
        L.orc_emc60.argtypes = [_f32p, C.c_int64, _f32p, _f32p, C.c_float, _u64p]
        L.orc_test_pairs.argtypes = [_f32p, _f32p, C.c_int64, _i32p, C.c_int, C.c_int, _f32p, _f32p, _f32p]
        L.orc_ploc.restype = C.c_int64
        L.orc_ploc.argtypes = [_f32p, C.c_int64, _i32p, C.c_void_p, C.c_int64, C.c_int, _i32p, _f32p, _i32p]
        L.orc_hploc.restype = C.c_int64
        L.orc_hploc.argtypes = [_f32p, C.c_int64, _i32p, _u64p, C.c_void_p, C.c_int, C.c_int, _i32p, _f32p, _i32p]
        L.orc_retrace_binary.argtypes = [_f32p, C.c_int64, _f32p, C.c_int32, _f32p, C.c_int64, C.c_int, _i64p, _i64p,
                                         _u8p, _i32p, _f32p]
        L.orc_shadow_rays.argtypes = [_f32p, _f32p, _i32p, _f32p, C.c_int64, C.c_int, _i32p, C.c_int, C.c_int, _f32p,
                                      C.c_int, C.c_uint32, _f32p]
        L.orc_hploc_boxes.restype = C.c_int64
        L.orc_hploc_boxes.argtypes = [_f32p, C.c_int64, _u64p, C.c_void_p, C.c_int, C.c_int, _i32p, _f32p, _i32p]
        L.orc_presplit.restype = C.c_int64
        L.orc_presplit.argtypes = [_f32p, C.c_int64, _i64p, C.c_int, C.c_int, _u32p, C.c_void_p, C.c_void_p]
        L.orc_ref_codes.argtypes = [_f32p, C.c_int64, _u32p, _i32p, _f32p, C.c_int64, C.c_int, _u64p]
        L.orc_pinhole_rays.argtypes = [_f32p, C.c_int, C.c_int, _f32p]
        L.orc_bounce_rays.argtypes = [_f32p, _f32p, _i32p, _f32p, C.c_int64, C.c_uint32, _f32p]

    def pinhole_rays(self, cam_pos, cam_dir, cam_up, fov, far, width, height):
        """Primary rays of the GPU frontend's pinhole generator, restated (records of 8 floats)."""
        cam = np.array([*cam_pos, *cam_dir, *cam_up, fov, far], dtype=np.float32)
        out = np.empty((width * height, 8), np.float32)
        self.lib.orc_pinhole_rays(cam, int(width), int(height), out)
        return out

    def bounce_rays(self, tris, rays, prim, t, seed):
        """Bounce rays of the GPU frontend's generator, restated (one per ray; misses get a null ray)."""
        tris, rays = _tris(tris), _rays(rays)
        prim = np.ascontiguousarray(prim, np.int32)
        t = np.ascontiguousarray(t, np.float32)
        out = np.empty((len(rays), 8), np.float32)
        self.lib.orc_bounce_rays(tris, rays, prim, t, len(rays), int(seed) & 0xFFFFFFFF, out)
        return out

    def shadow_rays(self, tris, rays, prim, t, width, area=(), samples=1, points=(), seed=42):
        """Shadow rays of the frontend's generator, restated (per hit: area lights x samples, then point lights)."""
        tris, rays = _tris(tris), _rays(rays)
        prim = np.ascontiguousarray(prim, np.int32)
        t = np.ascontiguousarray(t, np.float32)
        area = np.ascontiguousarray(np.asarray(area, np.int32).reshape(-1))
        points = np.ascontiguousarray(np.asarray(points, np.float32).reshape(-1))
        per_hit = len(area) * samples + len(points) // 3
        out = np.empty((len(rays) * per_hit, 8), np.float32)
        self.lib.orc_shadow_rays(tris, rays, prim, t, len(rays), int(width), area if len(area) else np.zeros(1, np.int32),
                                 len(area), int(samples), points if len(points) else np.zeros(3, np.float32),
                                 len(points) // 3, int(seed) & 0xFFFFFFFF, out)
        return out

    def set_threads(self, n):
        self.lib.orc_set_threads(int(n))

    def brute(self, tris, rays, leaf_test=0, backface=False):
        tris, rays = _tris(tris), _rays(rays)
        h = Hits(len(rays))
        self.lib.orc_brute_closest(tris, len(tris), rays, len(rays), int(leaf_test), int(backface), h.prim, h.t,
                                   h.u, h.v)
        return h

    def brute_any(self, tris, rays, leaf_test=0, backface=False):
        tris, rays = _tris(tris), _rays(rays)
        occ = np.empty(len(rays), np.uint8)
        self.lib.orc_brute_any(tris, len(tris), rays, len(rays), int(leaf_test), int(backface), occ)
        return occ.astype(bool)

    def test_pairs(self, tris, rays, prim, leaf_test=0, backface=False):
        """Leaf test of each ray against its own triangle prim[r] (t = +inf where prim < 0 or a miss)."""
        tris, rays = _tris(tris), _rays(rays)
        prim = np.ascontiguousarray(prim, np.int32)
        h = Hits(len(rays))
        h.prim = prim
        self.lib.orc_test_pairs(tris, rays, len(rays), prim, int(leaf_test), int(backface), h.t, h.u, h.v)
        return h

    def intersect_f64(self, tris, rays, prim):
        tris, rays = _tris(tris), _rays(rays)
        prim = np.ascontiguousarray(prim, np.int32)
        t, u, v = (np.empty(len(rays)) for _ in range(3))
        self.lib.orc_intersect_f64(tris, rays, len(rays), prim, t, u, v)
        return t, u, v

    def brute_f64(self, tris, rays):
        tris, rays = _tris(tris), _rays(rays)
        prim = np.empty(len(rays), np.int32)
        t = np.empty(len(rays))
        self.lib.orc_brute_closest_f64(tris, len(tris), rays, len(rays), prim, t)
        return prim, t

    def scene_bounds(self, tris):
        tris = _tris(tris)
        out = [np.empty(3, np.float32) for _ in range(4)]
        self.lib.orc_scene_bounds(tris, len(tris), *out)
        return out  # cmin, cmax, bmin, bmax

    def morton30(self, tris):
        tris = _tris(tris)
        cmin, cmax, _, _ = self.scene_bounds(tris)
        codes = np.empty(len(tris), np.uint32)
        self.lib.orc_morton30(tris, len(tris), cmin, cmax, codes)
        return codes

    def emc60(self, tris):
        tris = _tris(tris)
        cmin, cmax, bmin, bmax = self.scene_bounds(tris)
        diag = self.lib.orc_scene_diag(bmin, bmax)
        codes = np.empty(len(tris), np.uint64)
        self.lib.orc_emc60(tris, len(tris), cmin, cmax, diag, codes)
        return codes

    def emc60_plan(self, tris):
        cmin, cmax, bmin, bmax = self.scene_bounds(tris)
        diag = self.lib.orc_scene_diag(bmin, bmax)
        bits = np.empty(4, np.int32)
        masks = np.empty(4, np.uint64)
        self.lib.orc_emc60_plan(cmin, cmax, diag, bits, masks)
        return bits, masks

    def hploc(self, tris, perm, sorted_keys, radius=16, seg=None, threshold=16):
        """Hierarchical PLOC over the radix tree of the sorted keys (orc_hploc). Returns (children (n-1, 2) int32,
        boxes (n-1, 6) float32, iterations): row k is internal node id n + k; rows of the splits between segments
        stay unused (-1 children)."""
        tris = _tris(tris)
        perm = np.ascontiguousarray(perm, np.int32)
        keys = np.ascontiguousarray(sorted_keys).astype(np.uint64)
        n = len(tris)
        rows = max(n - 1, 1)
        children = np.full(2 * rows, -1, np.int32)
        boxes = np.zeros(6 * rows, np.float32)
        it = np.zeros(1, np.int32)
        seg_arr = None if seg is None else np.ascontiguousarray(seg, np.int32)
        segp = None if seg_arr is None else seg_arr.ctypes.data_as(C.c_void_p)
        k = self.lib.orc_hploc(tris, n, perm, keys, segp, int(radius), int(threshold), children, boxes, it)
        if k < 0:
            raise ValueError("orc_hploc: bad input")
        return children[: 2 * (n - 1)].reshape(-1, 2), boxes[: 6 * (n - 1)].reshape(-1, 6), int(it[0])

    def retrace_binary(self, nodes, tris, root, rays, backface=False):
        """Re-traversal of a downloaded binary layout (orc_retrace_binary): per ray (visits, tests, stable, prim, t).
        ``nodes`` are the layout's bytes (64 per node), ``tris`` its leaf triangles (N, 3, 4) float32."""
        nodes = np.ascontiguousarray(np.frombuffer(np.ascontiguousarray(nodes).tobytes(), np.float32))
        tris = np.ascontiguousarray(tris, np.float32).reshape(-1)
        rays = _rays(rays)
        n = len(rays)
        visits, tests = np.zeros(n, np.int64), np.zeros(n, np.int64)
        stable = np.zeros(n, np.uint8)
        prim, t = np.zeros(n, np.int32), np.zeros(n, np.float32)
        self.lib.orc_retrace_binary(nodes, len(nodes) // 16, tris, int(root), rays, n, int(backface), visits, tests,
                                    stable, prim, t)
        return visits, tests, stable.astype(bool), prim, t

    def presplit(self, tris, budget, mesh_sizes=None):
        """Pre-splitting of large triangles (orc_presplit): (pieces per triangle, ref_tri (R,), ref boxes (R, 6))."""
        tris = _tris(tris)
        sizes = np.ascontiguousarray([len(tris)] if mesh_sizes is None else mesh_sizes, np.int64)
        pieces = np.zeros(len(tris), np.uint32)
        total = self.lib.orc_presplit(tris, len(tris), sizes, len(sizes), int(budget), pieces, None, None)
        ref_tri = np.zeros(max(total, 1), np.int32)
        rbox = np.zeros((max(total, 1), 6), np.float32)
        self.lib.orc_presplit(tris, len(tris), sizes, len(sizes), int(budget), pieces,
                              ref_tri.ctypes.data_as(C.c_void_p), rbox.ctypes.data_as(C.c_void_p))
        return pieces, ref_tri[:total], rbox[:total]

    def ref_codes(self, tris, pieces, ref_tri, rbox, code_type):
        """Codes of one mesh's references (orc_ref_codes): 0 Morton30 (in uint64), 1 EMC60."""
        tris = _tris(tris)
        codes = np.zeros(len(ref_tri), np.uint64)
        self.lib.orc_ref_codes(tris, len(tris), np.ascontiguousarray(pieces, np.uint32),
                               np.ascontiguousarray(ref_tri, np.int32), np.ascontiguousarray(rbox, np.float32),
                               len(ref_tri), int(code_type), codes)
        return codes

    def hploc_boxes(self, leaf_boxes, sorted_keys, radius=16, threshold=16):
        """orc_hploc over given leaf boxes in sorted order (e.g. pre-split references)."""
        lb = np.ascontiguousarray(leaf_boxes, np.float32)
        n = len(lb)
        rows = max(n - 1, 1)
        children = np.full(2 * rows, -1, np.int32)
        boxes = np.zeros(6 * rows, np.float32)
        it = np.zeros(1, np.int32)
        k = self.lib.orc_hploc_boxes(lb, n, np.ascontiguousarray(sorted_keys).astype(np.uint64), None, int(radius),
                                     int(threshold), children, boxes, it)
        if k < 0:
            raise ValueError("orc_hploc_boxes: bad input")
        return children[: 2 * (n - 1)].reshape(-1, 2), boxes[: 6 * (n - 1)].reshape(-1, 6), int(it[0])

    def ploc(self, tris, perm, radius=16, seg=None, nseg=1):
        """Returns (children (K,2) int32, boxes (K,6) float32, iterations)."""
        tris = _tris(tris)
        perm = np.ascontiguousarray(perm, np.int32)
        n = len(tris)
        k_max = max(n - nseg, 0)
        children = np.empty(2 * max(k_max, 1), np.int32)
        boxes = np.empty(6 * max(k_max, 1), np.float32)
        it = np.zeros(1, np.int32)
        seg_arr = None if seg is None else np.ascontiguousarray(seg, np.int32)
        segp = None if seg_arr is None else seg_arr.ctypes.data_as(C.c_void_p)
        k = self.lib.orc_ploc(tris, n, perm, segp, int(nseg), int(radius), children, boxes, it)
        if k < 0:
            raise ValueError("orc_ploc: bad input")
        return children[: 2 * k].reshape(-1, 2), boxes[: 6 * k].reshape(-1, 6), int(it[0])


def classify_hits(prim, t, u, v, brute, sbvh=None):
    """Agreement classes of GPU closest hits (ref_mt leaf test) against the reference's brute force and SBvh.

    Against brute force: E = id, t, u and v bit-equal; T = a different id at a bit-equal t (an exact tie broken
    another way); F = anything else. Against SBvh (optional): same = equal id; S = SBvh differs, the GPU record
    is brute force's (E) and SBvh's t is not nearer (SBvh missed, took a farther hit or broke a tie by traversal
    order: its bounds are not conservative); F = any other difference."""
    def b(a):
        return np.ascontiguousarray(a, np.float32).view(np.uint32)
    prim = np.asarray(prim)
    same_id = prim == brute.prim
    same_t = b(t) == b(brute.t)
    exact = same_id & same_t & (b(u) == b(brute.u)) & (b(v) == b(brute.v))
    tie = ~same_id & same_t & (prim >= 0)
    out = {"rays": int(len(prim)), "E": int(exact.sum()), "T": int(tie.sum()), "F": int((~exact & ~tie).sum())}
    if sbvh is not None:
        diff = prim != sbvh.prim
        sb_t = np.where(sbvh.prim >= 0, sbvh.t, np.inf)
        gt = np.where(prim >= 0, np.asarray(t, np.float32), np.inf)
        s_cls = diff & exact & (sb_t >= gt)
        out["vs_sbvh"] = {"same_id": int((~diff).sum()), "S": int(s_cls.sum()), "F": int((diff & ~s_cls).sum())}
    return out


def sort_perm(codes, seg=None):
    """Stable order of the codes (ties keep triangle order), optionally by (segment, code)."""
    if seg is None:
        return np.argsort(codes, kind="stable").astype(np.int32)
    return np.lexsort((codes, seg)).astype(np.int32)


def sah_cost_binary(children, boxes, n_leaves, leaf_boxes, max_leaf_exclusive=4):
    """FP64 SAH cost of a clustering tree after the leaf rule "a node with < L triangles is a leaf". Row k of
    children/boxes is internal node n_leaves + k (rows with children -1 are unused); the root is the one node that
    is nobody's child."""
    k = len(children)
    if n_leaves == 1:
        return 1.0
    used = children[:, 0] >= 0
    is_child = np.zeros(n_leaves + k, bool)
    is_child[children[used].ravel()] = True
    roots = [n_leaves + i for i in np.nonzero(used)[0] if not is_child[n_leaves + i]]
    assert len(roots) == 1, roots
    root = roots[0]
    order, stack = [], [root]
    while stack:  # parents before children
        x = stack.pop()
        order.append(x)
        if x >= n_leaves:
            stack.extend(children[x - n_leaves].tolist())
    count = np.zeros(n_leaves + k, np.int64)
    for x in reversed(order):
        count[x] = 1 if x < n_leaves else count[children[x - n_leaves][0]] + count[children[x - n_leaves][1]]

    def sa(b):
        d = b[3:6].astype(np.float64) - b[0:3].astype(np.float64)
        return 2.0 * (d[0] * d[1] + d[1] * d[2] + d[2] * d[0])

    total = 0.0
    stack = [root]
    while stack:
        x = stack.pop()
        if x < n_leaves:
            total += sa(leaf_boxes[x])
            continue
        b = boxes[x - n_leaves]
        if count[x] < max_leaf_exclusive:
            total += sa(b) * count[x]
            continue
        total += sa(b)
        stack.extend(children[x - n_leaves].tolist())
    return total / sa(boxes[root - n_leaves])
