"""Host-side mirror of the reference's acceleration-structure interface, on top of the C ABI.

The reference's boundary (src/acceleration/acceleration_structure.h:12-19) is

    class AccelerationStructure {
        void Build(const AccelerationStructureConfig&, Stats&, std::span<const Triangle>);
        bool Intersect(Stats&, const Ray&, RayHit&, bool backface_culling) const;
        bool IntersectAny(Stats&, const Ray&, bool backface_culling) const;
    };

created by ``CreateAccelerationStucture(config)`` (acceleration_structure_factory.cc:9-19) from an
``AccelerationStructureConfig`` (src/config/acceleration_structure_config.h:9-29). ``GpuPlocBvh`` keeps the
same names, argument meaning and error behaviour, batched: ``Intersect`` takes a whole ray batch and
returns hit records (prim, t, u = b1, v = b2) instead of filling one ``RayHit``. Device memory and streams
come from PyTorch; every computation runs in libdipl_bvh.so.
"""
from __future__ import annotations

import ctypes as C
import enum
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib as L


class AccelerationStructureType(enum.Enum):
    """The reference enum (acceleration_structure_config.h:9); the PLOC kinds are built by this engine."""
    kDummy = "dummy"
    kSbvh = "sbvh"
    kPloc = "ploc"
    kPlocEmc = "ploc_emc"
    kPlocSobb = "ploc_sobb"
    kPlocEmcSobb = "ploc_emc_sobb"


def parse_acceleration_structure_type(s: str) -> AccelerationStructureType:
    """ParseEnum<AccelerationStructureType> (acceleration_structure_config.h:12-20): RuntimeError if invalid."""
    for t in AccelerationStructureType:
        if t.value == s:
            return t
    raise RuntimeError("Invalid AccelerationStructureType: " + s)


# Bridge of the PLOC kinds to (code, bounding volume): BridgeAccelerationConfig, src/gpu/config/gpu_config_bridge.cc:24-60.
_BRIDGE = {
    AccelerationStructureType.kPloc: (L.CODE_MORTON30, L.BV_AABB),
    AccelerationStructureType.kPlocEmc: (L.CODE_EMC60, L.BV_AABB),
    AccelerationStructureType.kPlocSobb: (L.CODE_MORTON30, L.BV_SOBB),
    AccelerationStructureType.kPlocEmcSobb: (L.CODE_EMC60, L.BV_SOBB),
}


@dataclass
class AccelerationStructureConfig:
    """Reference fields (acceleration_structure_config.h:22-29) plus this engine's options."""
    acceleration_structure_type: AccelerationStructureType = AccelerationStructureType.kPloc
    max_depth: int = 32
    nn_search_radius: int = 16          # PLOC radius (reference default 10; the workloads use 16)
    kdop_size: int = 32
    max_triangles_per_leaf: int = 4     # a node with fewer triangles is a leaf (sbvh.cc:273-276)
    bin_count: int = 16
    layout: str = "binary"              # "binary" | "wide8_q8"
    leaf_test: str = "ref_mt"           # "ref_mt" | "watertight"
    ploc_block_size: int = 0
    sort_digit_bits: int = 0
    clustering: str = "hploc"           # "hploc" (hierarchical, default) | "ploc" (global iterations)
    split_budget: int = 0               # pre-splitting of large triangles: at most this % more leaves (0 = none)


@dataclass
class AccelerationStats:
    """The reference's AccelerationStats (src/stats/acceleration_stats.h:5-17), with 64-bit Python ints."""
    build_time: float = 0.0
    node_count: int = 0
    inner_node_count: int = 0
    leaf_node_count: int = 0
    memory_consumption: int = 0
    query_count: int = 0
    intersection_count: int = 0
    traversal_count: int = 0


@dataclass
class RaytracingStats:
    """The reference's RaytracingStats (src/stats/raytracing_stats.h:5-10): seconds and ray counts of a frame.
    ``trace_frame`` fills it the way CpuRaytracer does (cpu_raytracer.cc:88-147): one primary ray per pixel, one
    secondary ray per traced bounce."""
    raytracing_time: float = 0.0
    primary_ray_count: int = 0
    secondary_ray_count: int = 0
    shadow_ray_count: int = 0


@dataclass
class Stats:
    """The reference's Stats (src/stats/stats.h:8-11)."""
    rt_stats: RaytracingStats = field(default_factory=RaytracingStats)
    accel_stats: AccelerationStats = field(default_factory=AccelerationStats)


@dataclass
class Hits:
    """Closest-hit records: prim (int32, -1 = miss), t (+inf on a miss), u = b1, v = b2 (device tensors)."""
    prim: torch.Tensor
    t: torch.Tensor
    u: torch.Tensor
    v: torch.Tensor
    raw: torch.Tensor  # (R, 4) int32 view of the dipl_hit records


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t: torch.Tensor):
    return C.c_void_p(t.data_ptr()) if t is not None and t.numel() > 0 else C.c_void_p(0)


def _leaf_test(name: str) -> int:
    if name == "ref_mt":
        return L.LEAF_REF_MT
    if name == "watertight":
        return L.LEAF_WATERTIGHT
    raise ValueError(f"unknown leaf test {name!r}")


def soa_vertices(triangles, device="cuda"):
    """(N, 3, 3) float32 triangles -> three contiguous (N, 3) device tensors (tri_v0/v1/v2_pos layout)."""
    if isinstance(triangles, np.ndarray):
        triangles = torch.from_numpy(np.ascontiguousarray(triangles, dtype=np.float32))
    if triangles.dtype != torch.float32 or triangles.dim() != 3 or tuple(triangles.shape[1:]) != (3, 3):
        raise ValueError("triangles must be float32 of shape (N, 3, 3)")
    triangles = triangles.to(device)
    return tuple(triangles[:, k, :].contiguous() for k in range(3))


def as_device_rays(rays, device="cuda") -> torch.Tensor:
    if isinstance(rays, np.ndarray):
        rays = torch.from_numpy(np.ascontiguousarray(rays, dtype=np.float32))
    if rays.dtype != torch.float32 or rays.dim() != 2 or rays.shape[1] != 8:
        raise ValueError("rays must be float32 of shape (R, 8): origin, tmin, direction, tmax")
    return rays.to(device).contiguous()


def make_desc(v0, v1, v2, config: AccelerationStructureConfig) -> L.BuildDesc:
    kind = config.acceleration_structure_type
    if kind not in _BRIDGE:
        # the reference factory throws std::invalid_argument for kinds it cannot create (factory.cc:17)
        raise ValueError(f"{kind.value} is not a GPU PLOC acceleration structure")
    code, bv = _BRIDGE[kind]
    d = L.default_desc()
    n = v0.shape[0]
    d.d_v0, d.d_v1, d.d_v2 = (t.data_ptr() if n else None for t in (v0, v1, v2))
    d.num_triangles = n
    d.code_type, d.bv_type = code, bv
    d.layout = {"binary": L.LAYOUT_BINARY, "wide8_q8": L.LAYOUT_WIDE8_Q8}[config.layout]
    d.max_triangles_per_leaf = config.max_triangles_per_leaf
    d.nn_search_radius = config.nn_search_radius
    d.kdop_size = config.kdop_size
    d.ploc_block_size = config.ploc_block_size
    d.sort_digit_bits = config.sort_digit_bits
    d.clustering = {"hploc": L.CLUSTER_HPLOC, "ploc": L.CLUSTER_PLOC}[config.clustering]
    d.split_budget = config.split_budget
    return d


class GpuPlocBvh:
    """PLOC BVH on the GPU behind the reference's AccelerationStructure interface (batched rays)."""

    def __init__(self):
        self._lib = L.load()
        self._h = C.c_void_p(0)
        self.config = None
        self.num_triangles = 0

    # -- AccelerationStructure::Build -------------------------------------------------------------
    def Build(self, acceleration_structure_config: AccelerationStructureConfig, stats: Stats, triangles):
        """Builds over (N, 3, 3) float32 triangles (torch tensor on any device, or numpy)."""
        self.close()
        self.config = acceleration_structure_config
        self._v = soa_vertices(triangles)  # kept for the adjoint and FP64 re-intersection
        d = make_desc(*self._v, acceleration_structure_config)
        t0 = time.perf_counter()
        L.check(self._lib.dipl_bvh_build(C.byref(d), C.byref(self._h), _stream()), "dipl_bvh_build")
        stats.accel_stats.build_time = (time.perf_counter() - t0) * 1e3
        self.num_triangles = d.num_triangles
        info = self.info()
        stats.accel_stats.inner_node_count = int(info.num_inner_nodes)
        stats.accel_stats.node_count = int(info.num_inner_nodes) * 2 + 1
        stats.accel_stats.leaf_node_count = stats.accel_stats.node_count - int(info.num_inner_nodes)
        stats.accel_stats.memory_consumption = int(info.node_bytes + info.triangle_bytes)
        return self

    @classmethod
    def from_handle(cls, handle, v, config):
        obj = cls()
        obj._h = handle
        obj._v = v
        obj.config = config
        obj.num_triangles = v[0].shape[0]
        return obj

    # -- AccelerationStructure::Intersect (batched) ---------------------------------------------------
    def Intersect(self, stats: Stats, rays, backface_culling: bool = False, leaf_test: str | None = None,
                  count: bool = False, coherent_order: bool = False) -> Hits:
        """Closest hits of a ray batch. With ``coherent_order``, a batch of 2^20 rays or more is traced in an order
        sorted on the device by origin cell and direction octant; the records are the same either way."""
        rays = as_device_rays(rays)
        n = rays.shape[0]
        raw = torch.empty((n, 4), dtype=torch.int32, device=rays.device)
        flags = (L.TRACE_BACKFACE_CULLING if backface_culling else 0) | (L.TRACE_COHERENT_ORDER if coherent_order else 0)
        lt = _leaf_test(leaf_test or self.config.leaf_test)
        if count:
            ctr = torch.zeros(2, dtype=torch.int64, device=rays.device)
            L.check(self._lib.dipl_bvh_trace_closest_counted(self._h, _ptr(rays), n, _ptr(raw), lt, flags, _ptr(ctr),
                                                             _stream()), "dipl_bvh_trace_closest_counted")
            c = ctr.cpu().tolist()
            stats.accel_stats.traversal_count += c[0]
            stats.accel_stats.intersection_count += c[1]
        else:
            L.check(self._lib.dipl_bvh_trace_closest(self._h, _ptr(rays), n, _ptr(raw), lt, flags, _stream()),
                    "dipl_bvh_trace_closest")
        stats.accel_stats.query_count += n
        f = raw.view(torch.float32)
        return Hits(raw[:, 0], f[:, 1], f[:, 2], f[:, 3], raw)

    # -- AccelerationStructure::IntersectAny (batched) ------------------------------------------------
    def IntersectAny(self, stats: Stats, rays, backface_culling: bool = False,
                     leaf_test: str | None = None) -> torch.Tensor:
        rays = as_device_rays(rays)
        n = rays.shape[0]
        occ = torch.empty(n, dtype=torch.uint8, device=rays.device)
        flags = L.TRACE_BACKFACE_CULLING if backface_culling else 0
        lt = _leaf_test(leaf_test or self.config.leaf_test)
        L.check(self._lib.dipl_bvh_trace_any(self._h, _ptr(rays), n, _ptr(occ), lt, flags, _stream()),
                "dipl_bvh_trace_any")
        stats.accel_stats.query_count += n
        return occ.bool()

    # -- extras -----------------------------------------------------------------------------------
    def info(self) -> L.BvhInfo:
        info = L.BvhInfo()
        L.check(self._lib.dipl_bvh_get_info(self._h, C.byref(info)), "dipl_bvh_get_info")
        return info

    def check_errors(self):
        """Raises DiplError if a trace on this BVH recorded a device-side failure (synchronises)."""
        L.check(self._lib.dipl_bvh_check_errors(self._h, _stream()), "dipl_bvh_check_errors")

    def sah_cost(self) -> float:
        c = C.c_double(0.0)
        L.check(self._lib.dipl_bvh_sah_cost(self._h, C.byref(c), _stream()), "dipl_bvh_sah_cost")
        return c.value

    def download_topology(self):
        """(perm (n,), children (n-1, 2), boxes (n-1, 6)) of the clustering, as numpy arrays; n = the clustering's
        leaves (the triangles, and their pieces with pre-splitting)."""
        n = int(self.info().num_leaves)
        perm = np.empty(max(n, 1), np.int32)
        ch = np.empty(max(2 * (n - 1), 1), np.int32)
        bx = np.empty(max(6 * (n - 1), 1), np.float32)
        L.check(self._lib.dipl_bvh_download_topology(self._h, perm.ctypes.data, ch.ctypes.data, bx.ctypes.data,
                                                     _stream()), "dipl_bvh_download_topology")
        k = max(n - 1, 0)
        return perm[:n], ch[: 2 * k].reshape(k, 2), bx[: 6 * k].reshape(k, 6)

    def download_layout(self):
        """(nodes bytes as uint8 array, triangles (N, 3, 4) float32, root reference)."""
        info = self.info()
        nodes = np.empty(max(int(info.node_bytes), 1), np.uint8)
        nl = int(info.num_leaves)
        tris = np.empty((max(nl, 1), 3, 4), np.float32)
        root = C.c_int32(0)
        L.check(self._lib.dipl_bvh_download_layout(self._h, nodes.ctypes.data, tris.ctypes.data, C.byref(root),
                                                   _stream()), "dipl_bvh_download_layout")
        return nodes[: int(info.node_bytes)], tris[:nl], root.value

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            L.check(self._lib.dipl_bvh_destroy(self._h), "dipl_bvh_destroy")
            self._h = C.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def CreateAccelerationStucture(config: AccelerationStructureConfig) -> GpuPlocBvh:
    """The reference factory (acceleration_structure_factory.cc:9-19), spelling kept; PLOC kinds only."""
    if config.acceleration_structure_type in _BRIDGE:
        return GpuPlocBvh()
    raise ValueError("Unkown AccelerationStructureType")


def build_batched(config: AccelerationStructureConfig, meshes, stats: Stats | None = None):
    """Builds one BVH per mesh in one pipeline (dipl_bvh_build_batched); returns a list of GpuPlocBvh."""
    lib = L.load()
    verts = [soa_vertices(m) for m in meshes]
    descs = (L.BuildDesc * len(meshes))()
    for i, v in enumerate(verts):
        descs[i] = make_desc(*v, config)
    handles = (C.c_void_p * len(meshes))()
    t0 = time.perf_counter()
    L.check(lib.dipl_bvh_build_batched(descs, len(meshes), handles, _stream()), "dipl_bvh_build_batched")
    if stats is not None:
        stats.accel_stats.build_time = (time.perf_counter() - t0) * 1e3
    return [GpuPlocBvh.from_handle(C.c_void_p(handles[i]), verts[i], config) for i in range(len(meshes))]


# -- building blocks ---------------------------------------------------------------------------------
def compute_codes(triangles, code_type=L.CODE_MORTON30) -> torch.Tensor:
    lib = L.load()
    v = soa_vertices(triangles)
    cfg = AccelerationStructureConfig(
        acceleration_structure_type=AccelerationStructureType.kPloc if code_type == L.CODE_MORTON30
        else AccelerationStructureType.kPlocEmc)
    d = make_desc(*v, cfg)
    n = v[0].shape[0]
    out = torch.empty(n, dtype=torch.int32 if code_type == L.CODE_MORTON30 else torch.int64, device=v[0].device)
    L.check(lib.dipl_compute_codes(C.byref(d), _ptr(out), _stream()), "dipl_compute_codes")
    return out


def radix_sort_pairs(keys: torch.Tensor, vals: torch.Tensor | None = None, begin_bit=0, end_bit=None,
                     digit_bits=0):
    """Stable LSD sort of int32/int64 (read as unsigned) keys with int32 values (default: 0..n-1)."""
    lib = L.load()
    kb = keys.element_size()
    end_bit = 8 * kb if end_bit is None else end_bit
    n = keys.numel()
    ko = torch.empty_like(keys)
    vo = torch.empty(n, dtype=torch.int32, device=keys.device)
    L.check(lib.dipl_radix_sort_pairs(_ptr(keys), _ptr(vals), _ptr(ko), _ptr(vo), n, kb, begin_bit, end_bit,
                                      digit_bits, _stream()), "dipl_radix_sort_pairs")
    return ko, vo


def reintersect_f64(v, rays: torch.Tensor, hits: Hits) -> torch.Tensor:
    lib = L.load()
    n = rays.shape[0]
    out = torch.empty((n, 3), dtype=torch.float64, device=rays.device)
    L.check(lib.dipl_reintersect_f64(_ptr(v[0]), _ptr(v[1]), _ptr(v[2]), _ptr(rays), _ptr(hits.raw), n, _ptr(out),
                                     _stream()), "dipl_reintersect_f64")
    return out


def trace_adjoint(v, rays: torch.Tensor, hits: Hits, dtuv: torch.Tensor):
    """Returns (dv0, dv1, dv2, dorig, ddir) for upstream gradients dtuv (R, 3)."""
    lib = L.load()
    n = rays.shape[0]
    dv = [torch.zeros_like(x) for x in v]
    dorig = torch.empty((n, 3), dtype=torch.float32, device=rays.device)
    ddir = torch.empty((n, 3), dtype=torch.float32, device=rays.device)
    dtuv = dtuv.to(torch.float32).contiguous()
    L.check(lib.dipl_trace_adjoint(_ptr(v[0]), _ptr(v[1]), _ptr(v[2]), _ptr(rays), _ptr(hits.raw), _ptr(dtuv), n,
                                   _ptr(dv[0]), _ptr(dv[1]), _ptr(dv[2]), _ptr(dorig), _ptr(ddir), _stream()),
            "dipl_trace_adjoint")
    return dv[0], dv[1], dv[2], dorig, ddir


# -- GPU frontend: wavefront ray generation (generate -> trace -> bounce -> trace) ---------------------------
def generate_pinhole_rays(cam_pos, cam_dir, cam_up, fov, far, width, height, device="cuda") -> torch.Tensor:
    """One primary ray per pixel (row-major from the top-left), generated on the device (dipl_generate_pinhole_rays)."""
    lib = L.load()
    cam = L.Camera((C.c_float * 3)(*cam_pos), (C.c_float * 3)(*cam_dir), (C.c_float * 3)(*cam_up), float(fov),
                   float(far))
    rays = torch.empty((width * height, 8), dtype=torch.float32, device=device)
    L.check(lib.dipl_generate_pinhole_rays(C.byref(cam), int(width), int(height), _ptr(rays), _stream()),
            "dipl_generate_pinhole_rays")
    return rays


def generate_bounce_rays(v, rays: torch.Tensor, hits: Hits, seed: int) -> torch.Tensor:
    """One cosine-weighted bounce ray per hit, on the device (dipl_generate_bounce_rays); misses get a ray that
    hits nothing. ``v`` are the SoA vertex arrays the BVH was built from."""
    lib = L.load()
    n = rays.shape[0]
    out = torch.empty_like(rays)
    L.check(lib.dipl_generate_bounce_rays(_ptr(v[0]), _ptr(v[1]), _ptr(v[2]), _ptr(rays), _ptr(hits.raw), n,
                                          int(seed) & 0xFFFFFFFF, _ptr(out), _stream()), "dipl_generate_bounce_rays")
    return out


def generate_shadow_rays(v, rays: torch.Tensor, hits: Hits, width: int, area_light_triangles=(), samples: int = 1,
                         point_lights=(), seed: int = 42) -> torch.Tensor:
    """Shadow rays of every hit toward the lights (dipl_generate_shadow_rays): (R * per_hit, 8), per_hit = area
    lights x samples + point lights, in the reference's light order; null rays where the reference casts none."""
    lib = L.load()
    n = rays.shape[0]
    dev = rays.device
    area = torch.as_tensor(np.asarray(area_light_triangles, np.int32).reshape(-1), device=dev)
    points = torch.as_tensor(np.asarray(point_lights, np.float32).reshape(-1, 3), device=dev).contiguous()
    per_hit = area.numel() * samples + points.shape[0]
    out = torch.empty((n * per_hit, 8), dtype=torch.float32, device=dev)
    L.check(lib.dipl_generate_shadow_rays(_ptr(v[0]), _ptr(v[1]), _ptr(v[2]), _ptr(rays), _ptr(hits.raw), n,
                                          int(width), _ptr(area), int(area.numel()), int(samples), _ptr(points),
                                          int(points.shape[0]), int(seed) & 0xFFFFFFFF, _ptr(out), _stream()),
            "dipl_generate_shadow_rays")
    return out


@dataclass
class Lights:
    """The lights of a frame's shadow wave: area lights (triangle ids) sampled ``samples`` times each (the reference
    RenderConfig's area_light_sample_cnt) and point lights (positions)."""
    area_light_triangles: tuple = ()
    samples: int = 1
    point_lights: tuple = ()
    seed: int = 42  # the reference's area-light sampling seed (cpu_raytracer.cc:181-182)


def trace_frame(bvh: "GpuPlocBvh", camera: dict, width: int, height: int, seed: int, stats: "Stats | None" = None,
                lights: "Lights | None" = None):
    """One wavefront frame of the renderer path: primary rays, their closest hits, one bounce ray per hit and
    the bounce hits, all on the device. Returns (primary rays, primary hits, bounce rays, bounce hits); with
    ``lights``, also (shadow rays, occluded flags) of the primary hits' shadow wave (IsShadowed through
    dipl_bvh_trace_any).

    With ``stats``, adds the frame to its RaytracingStats (time in seconds, synchronised; width * height primary
    rays; one secondary ray per primary hit, the bounces that carry a ray; one shadow ray per cast shadow ray) and its
    AccelerationStats queries."""
    st = stats if stats is not None else Stats()
    t0 = time.perf_counter()
    rays = generate_pinhole_rays(camera["cam_pos"], camera["cam_dir"], camera["cam_up"], camera["fov"],
                                 camera["far"], width, height)
    hits = bvh.Intersect(st, rays)
    bounce = generate_bounce_rays(bvh._v, rays, hits, seed)
    bhits = bvh.Intersect(st, bounce)
    shadow = occluded = None
    if lights is not None:
        shadow = generate_shadow_rays(bvh._v, rays, hits, width, lights.area_light_triangles, lights.samples,
                                      lights.point_lights, lights.seed)
        occluded = bvh.IntersectAny(st, shadow)
    if stats is not None:
        secondary = int((hits.prim >= 0).sum().item())  # synchronises the stream
        stats.rt_stats.raytracing_time += time.perf_counter() - t0
        stats.rt_stats.primary_ray_count += int(width) * int(height)
        stats.rt_stats.secondary_ray_count += secondary
        if shadow is not None:
            stats.rt_stats.shadow_ray_count += int((shadow[:, 7] > 0).sum().item())
    if lights is not None:
        return rays, hits, bounce, bhits, shadow, occluded
    return rays, hits, bounce, bhits


class BuildPlan:
    """A batch of meshes captured once into a CUDA graph (dipl_build_plan_*); ``launch`` rebuilds every BVH from
    the current vertex contents; ``bvhs`` waits and returns one GpuPlocBvh per mesh for the latest build."""

    def __init__(self, config: AccelerationStructureConfig, meshes, tuned_descs=None):
        self._lib = L.load()
        self.config = config
        self.verts = [soa_vertices(m) for m in meshes]
        n = len(self.verts)
        self.descs = (L.BuildDesc * n)()
        for i, v in enumerate(self.verts):
            self.descs[i] = make_desc(*v, config)
            if tuned_descs is not None:  # take the tuned knobs, keep this plan's own vertex arrays
                t = tuned_descs[i]
                self.descs[i].nn_search_radius = t.nn_search_radius
                self.descs[i].ploc_block_size = t.ploc_block_size
                self.descs[i].sort_digit_bits = t.sort_digit_bits
        self._h = C.c_void_p(0)
        L.check(self._lib.dipl_build_plan_create(self.descs, n, C.byref(self._h), _stream()), "dipl_build_plan_create")

    def launch(self):
        L.check(self._lib.dipl_build_plan_launch(self._h, _stream()), "dipl_build_plan_launch")

    def bvhs(self):
        n = len(self.verts)
        handles = (C.c_void_p * n)()
        L.check(self._lib.dipl_build_plan_get_bvhs(self._h, handles, _stream()), "dipl_build_plan_get_bvhs")
        return [GpuPlocBvh.from_handle(C.c_void_p(handles[i]), self.verts[i], self.config) for i in range(n)]

    def close(self):
        if self._h.value:
            self._lib.dipl_build_plan_destroy(self._h)
            self._h = C.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune(config: AccelerationStructureConfig, meshes, cache_path=None):
    """dipl_autotune_build over these meshes; returns (tuned descs array, from_cache)."""
    lib = L.load()
    verts = [soa_vertices(m) for m in meshes]
    n = len(verts)
    descs = (L.BuildDesc * n)()
    for i, v in enumerate(verts):
        descs[i] = make_desc(*v, config)
    tuned = (L.BuildDesc * n)()
    fc = C.c_int32(0)
    path = cache_path.encode() if cache_path else None
    L.check(lib.dipl_autotune_build(descs, n, path, tuned, C.byref(fc), _stream()), "dipl_autotune_build")
    return tuned, bool(fc.value), verts
