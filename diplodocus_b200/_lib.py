"""ctypes binding of libdipl_bvh.so (the C ABI declared in include/dipl_bvh.h).

The library is built in-tree (diplodocus_b200/lib/libdipl_bvh.so, see diplodocus_b200/build.py). There is
no fallback: if the library is missing or cannot be loaded, ``load()`` raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libdipl_bvh.so")

DIPL_OK = 0
STATUS = {0: "DIPL_OK", 1: "DIPL_ERR_INVALID_ARGUMENT", 2: "DIPL_ERR_CUDA", 3: "DIPL_ERR_OUT_OF_MEMORY",
          4: "DIPL_ERR_TIMEOUT", 5: "DIPL_ERR_INTERNAL", 6: "DIPL_ERR_UNSUPPORTED", 7: "DIPL_ERR_IO"}
DIPL_ERR_IO = 7

CODE_MORTON30, CODE_EMC60 = 0, 1
BV_AABB, BV_SOBB = 0, 1
LAYOUT_BINARY, LAYOUT_WIDE8_Q8 = 0, 1
LEAF_REF_MT, LEAF_WATERTIGHT = 0, 1
CLUSTER_HPLOC, CLUSTER_PLOC = 0, 1
TRACE_BACKFACE_CULLING = 1
TRACE_COHERENT_ORDER = 2

# Every entry point include/dipl_bvh.h declares.
EXPORTS = [
    "dipl_build_desc_init", "dipl_bvh_build", "dipl_bvh_build_batched", "dipl_build_plan_create",
    "dipl_build_plan_launch", "dipl_build_plan_get_bvhs", "dipl_build_plan_destroy", "dipl_autotune_build",
    "dipl_bvh_trace_closest",
    "dipl_bvh_trace_closest_counted", "dipl_bvh_trace_any", "dipl_bvh_sah_cost", "dipl_bvh_get_info",
    "dipl_bvh_download_topology", "dipl_bvh_download_layout", "dipl_bvh_check_errors", "dipl_bvh_destroy", "dipl_compute_codes",
    "dipl_radix_sort_pairs", "dipl_radix_sort_pairs_noalloc", "dipl_reintersect_f64", "dipl_trace_adjoint",
    "dipl_generate_pinhole_rays", "dipl_generate_bounce_rays", "dipl_generate_shadow_rays",
    "dipl_selftest_bounded_waits",
    "dipl_obj_scene_load", "dipl_obj_scene_get_info", "dipl_obj_scene_get_triangles", "dipl_obj_scene_get_soa",
    "dipl_obj_scene_get_materials", "dipl_obj_scene_get_lights", "dipl_obj_scene_destroy",
    "dipl_set_limits", "dipl_get_limits", "dipl_status_string",
    "dipl_last_error", "dipl_abi_version", "dipl_kernel_launch_count",
]


class BuildDesc(C.Structure):
    _fields_ = [("d_v0", C.c_void_p), ("d_v1", C.c_void_p), ("d_v2", C.c_void_p), ("num_triangles", C.c_int64),
                ("code_type", C.c_int32), ("bv_type", C.c_int32), ("layout", C.c_int32),
                ("max_triangles_per_leaf", C.c_int32), ("nn_search_radius", C.c_int32), ("kdop_size", C.c_int32),
                ("ploc_block_size", C.c_int32), ("sort_digit_bits", C.c_int32), ("clustering", C.c_int32),
                ("split_budget", C.c_int32)]


class BvhInfo(C.Structure):
    _fields_ = [("num_triangles", C.c_int64), ("num_inner_nodes", C.c_int64), ("num_leaves", C.c_int64),
                ("node_bytes", C.c_int64), ("triangle_bytes", C.c_int64), ("depth", C.c_int32),
                ("ploc_iterations", C.c_int32), ("code_type", C.c_int32), ("bv_type", C.c_int32),
                ("layout", C.c_int32), ("max_triangles_per_leaf", C.c_int32), ("nn_search_radius", C.c_int32),
                ("kdop_size", C.c_int32), ("clustering", C.c_int32), ("reserved", C.c_int32)]


class Limits(C.Structure):
    _fields_ = [("device_memory_bytes", C.c_uint64), ("clustering_iterations", C.c_uint32),
                ("trace_steps", C.c_uint32)]


class ObjSceneInfo(C.Structure):
    _fields_ = [("num_triangles", C.c_int64), ("num_materials", C.c_int64), ("num_area_lights", C.c_int64),
                ("num_point_lights", C.c_int64), ("camera", C.c_float * 11)]


class Camera(C.Structure):
    """dipl_camera: pinhole camera (pos, dir, up, fov in radians, far = primary rays' tmax)."""
    _fields_ = [("pos", C.c_float * 3), ("dir", C.c_float * 3), ("up", C.c_float * 3), ("fov", C.c_float),
                ("far_t", C.c_float)]


class DiplError(RuntimeError):
    def __init__(self, status, where, msg):
        super().__init__(f"{where}: {STATUS.get(status, status)}: {msg}")
        self.status = status


_lib = None


def load(path: str = LIB_PATH):
    """Load the engine library (once). Raises if it is missing: there is no CPU fallback."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing; build it with `python -m diplodocus_b200.build`")
    L = C.CDLL(path)
    vp, i64, i32, u32 = C.c_void_p, C.c_int64, C.c_int32, C.c_uint32
    sig = {
        "dipl_build_desc_init": (None, [C.POINTER(BuildDesc)]),
        "dipl_bvh_build": (i32, [C.POINTER(BuildDesc), C.POINTER(vp), vp]),
        "dipl_bvh_build_batched": (i32, [C.POINTER(BuildDesc), i32, C.POINTER(vp), vp]),
        "dipl_build_plan_create": (i32, [C.POINTER(BuildDesc), i32, C.POINTER(vp), vp]),
        "dipl_build_plan_launch": (i32, [vp, vp]),
        "dipl_build_plan_get_bvhs": (i32, [vp, C.POINTER(vp), vp]),
        "dipl_build_plan_destroy": (i32, [vp]),
        "dipl_autotune_build": (i32, [C.POINTER(BuildDesc), i32, C.c_char_p, C.POINTER(BuildDesc), C.POINTER(i32), vp]),
        "dipl_bvh_trace_closest": (i32, [vp, vp, i64, vp, i32, u32, vp]),
        "dipl_bvh_trace_closest_counted": (i32, [vp, vp, i64, vp, i32, u32, vp, vp]),
        "dipl_bvh_trace_any": (i32, [vp, vp, i64, vp, i32, u32, vp]),
        "dipl_bvh_sah_cost": (i32, [vp, C.POINTER(C.c_double), vp]),
        "dipl_bvh_get_info": (i32, [vp, C.POINTER(BvhInfo)]),
        "dipl_bvh_download_topology": (i32, [vp, vp, vp, vp, vp]),
        "dipl_bvh_download_layout": (i32, [vp, vp, vp, vp, vp]),
        "dipl_bvh_check_errors": (i32, [vp, vp]),
        "dipl_bvh_destroy": (i32, [vp]),
        "dipl_compute_codes": (i32, [C.POINTER(BuildDesc), vp, vp]),
        "dipl_radix_sort_pairs": (i32, [vp, vp, vp, vp, i64, i32, i32, i32, i32, vp]),
        "dipl_radix_sort_pairs_noalloc": (i32, [vp, vp, vp, vp, i64, i32, i32, i32, i32, vp]),
        "dipl_reintersect_f64": (i32, [vp, vp, vp, vp, vp, i64, vp, vp]),
        "dipl_trace_adjoint": (i32, [vp, vp, vp, vp, vp, vp, i64, vp, vp, vp, vp, vp, vp]),
        "dipl_generate_pinhole_rays": (i32, [C.POINTER(Camera), i32, i32, vp, vp]),
        "dipl_generate_bounce_rays": (i32, [vp, vp, vp, vp, vp, i64, u32, vp, vp]),
        "dipl_generate_shadow_rays": (i32, [vp, vp, vp, vp, vp, i64, i32, vp, i32, i32, vp, i32, u32, vp, vp]),
        "dipl_selftest_bounded_waits": (i32, [u32, vp, vp]),
        "dipl_obj_scene_load": (i32, [C.c_char_p, C.c_char_p, C.POINTER(C.c_void_p)]),
        "dipl_obj_scene_get_info": (i32, [vp, C.POINTER(ObjSceneInfo)]),
        "dipl_obj_scene_get_triangles": (i32, [vp, vp, vp, vp, vp, vp]),
        "dipl_obj_scene_get_soa": (i32, [vp, vp, vp, vp]),
        "dipl_obj_scene_get_materials": (i32, [vp, vp, vp]),
        "dipl_obj_scene_get_lights": (i32, [vp, vp, vp, vp, vp]),
        "dipl_obj_scene_destroy": (None, [vp]),
        "dipl_set_limits": (i32, [C.POINTER(Limits)]),
        "dipl_get_limits": (i32, [C.POINTER(Limits), C.POINTER(C.c_uint64)]),
        "dipl_status_string": (C.c_char_p, [i32]),
        "dipl_last_error": (C.c_char_p, []),
        "dipl_abi_version": (i32, []),
        "dipl_kernel_launch_count": (C.c_uint64, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(status, where):
    if status != DIPL_OK:
        msg = _lib.dipl_last_error().decode(errors="replace") if _lib else ""
        raise DiplError(status, where, msg)


def default_desc() -> BuildDesc:
    d = BuildDesc()
    load().dipl_build_desc_init(C.byref(d))
    return d


def get_limits():
    """(Limits, device bytes the library holds now)."""
    lim, used = Limits(), C.c_uint64(0)
    check(load().dipl_get_limits(C.byref(lim), C.byref(used)), "dipl_get_limits")
    return lim, used.value


def set_limits(device_memory_bytes=0, clustering_iterations=0, trace_steps=0):
    """Process-wide limits (dipl_set_limits); all zero restores the defaults."""
    lim = Limits(int(device_memory_bytes), int(clustering_iterations), int(trace_steps))
    check(load().dipl_set_limits(C.byref(lim)), "dipl_set_limits")
