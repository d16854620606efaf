"""OBJ scene path into the engine: the reference's ObjSceneLoader behind the library's C ABI, feeding device SoA.

``load_obj_scene`` calls ``dipl_obj_scene_load`` (csrc/scene_obj.cu), the host-side restatement of
``ObjSceneLoader::Load / LoadObj / LoadMetadata`` (src/io/scene/obj_scene_loader.cc:20-205) and of the parts of
its vendored tinyobjloader 2.0 that decide which triangles come out. Triangles come out in file order with the
reference Scene's float bits; geometric normals and area lights are the reference's. ``Scene.device_vertices``
gives the three SoA vertex arrays ``dipl_build_desc`` takes, and ``render_scene_frame`` runs a scene file ->
PLOC build -> wavefront frame on the device.
"""
from __future__ import annotations

import logging
from dataclasses import dataclass, field

import numpy as np

log = logging.getLogger(__name__)

F32 = np.float32


# ---------------------------------------------------------------------------------------------------------
# Scene types (src/scene/*.h)
# ---------------------------------------------------------------------------------------------------------
@dataclass
class Material:
    """src/scene/material.h: the MTL values the reference keeps."""
    name: str
    ambient: np.ndarray
    diffuse: np.ndarray
    specular: np.ndarray
    transmittance: np.ndarray
    emission: np.ndarray
    shininess: F32
    ior: F32
    r_ior: F32
    dissolve: F32


@dataclass
class PointLight:
    pos: np.ndarray
    color: np.ndarray
    power: F32


@dataclass
class AreaLight:
    """src/scene/light.h. The reference never sets ``power`` for OBJ area lights; it is 0 here."""
    color: np.ndarray
    triangle_id: int
    surface_area: F32
    power: F32 = F32(0.0)


@dataclass
class Camera:
    pos: np.ndarray = field(default_factory=lambda: np.zeros(3, F32))
    dir: np.ndarray = field(default_factory=lambda: np.zeros(3, F32))
    up: np.ndarray = field(default_factory=lambda: np.zeros(3, F32))
    fov: F32 = F32(0.0)
    far: F32 = F32(0.0)

    def as_dict(self) -> dict:
        """The camera as ``accel.trace_frame`` takes it."""
        return {"cam_pos": self.pos.tolist(), "cam_dir": self.dir.tolist(), "cam_up": self.up.tolist(),
                "fov": float(self.fov), "far": float(self.far)}


@dataclass
class Scene:
    """src/scene/scene.h, flattened: triangle i is positions[i] = (v0, v1, v2) xyz."""
    positions: np.ndarray            # (N, 9) float32
    normals: np.ndarray              # (N, 9) float32, zero where the triangle has no vertex normals
    has_vertex_normals: np.ndarray   # (N,) bool
    geom_normals: np.ndarray         # (N, 3) float32, Normalize(Cross(v1 - v0, v2 - v0))
    material_ids: np.ndarray         # (N,) int32, -1 = no material
    materials: list
    area_lights: list
    point_lights: list
    camera: Camera

    def __len__(self) -> int:
        return len(self.positions)

    def triangles(self) -> np.ndarray:
        """(N, 3, 3) float32 view, the layout the engine's scene helpers and the oracle take."""
        return self.positions.reshape(-1, 3, 3)

    def device_vertices(self, device="cuda"):
        """(v0, v1, v2) float3 SoA device arrays (the reference GPU scene's ``tri_v{0,1,2}_pos``)."""
        from . import accel
        return accel.soa_vertices(self.triangles(), device)


# ---------------------------------------------------------------------------------------------------------
# Loading: the library's native loader (dipl_obj_scene_*), copied into numpy
# ---------------------------------------------------------------------------------------------------------
def load_obj_scene(dirpath, name) -> Scene | None:
    """ObjSceneLoader::Load (obj_scene_loader.cc:189-205): ``<dirpath>/<name>.meta`` then ``<name>.obj`` and the
    MTL files it names, read by the library (``dipl_obj_scene_load``). None where the reference returns
    std::nullopt (the reason is logged)."""
    import ctypes as C

    from . import _lib as L
    lib = L.load()
    h = C.c_void_p(0)
    st = lib.dipl_obj_scene_load(str(dirpath).encode(), str(name).encode(), C.byref(h))
    if st == L.DIPL_ERR_IO:
        log.error("%s", lib.dipl_last_error().decode(errors="replace"))
        return None
    L.check(st, "dipl_obj_scene_load")
    try:
        info = L.ObjSceneInfo()
        L.check(lib.dipl_obj_scene_get_info(h, C.byref(info)), "dipl_obj_scene_get_info")
        n, nm, na, npl = info.num_triangles, info.num_materials, info.num_area_lights, info.num_point_lights
        pos = np.zeros((n, 9), F32)
        nrm = np.zeros((n, 9), F32)
        geom = np.zeros((n, 3), F32)
        mat = np.zeros(n, np.int32)
        has_n = np.zeros(n, np.uint8)
        ptr = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
        L.check(lib.dipl_obj_scene_get_triangles(h, ptr(pos), ptr(nrm), ptr(geom), ptr(mat), ptr(has_n)),
                "dipl_obj_scene_get_triangles")
        mvals = np.zeros((nm, 19), F32)
        names = np.zeros((nm, 64), np.uint8)
        L.check(lib.dipl_obj_scene_get_materials(h, ptr(mvals), ptr(names)), "dipl_obj_scene_get_materials")
        al_id = np.zeros(na, np.int32)
        al_color = np.zeros((na, 3), F32)
        al_area = np.zeros(na, F32)
        pls = np.zeros((npl, 7), F32)
        L.check(lib.dipl_obj_scene_get_lights(h, ptr(al_id), ptr(al_color), ptr(al_area), ptr(pls)),
                "dipl_obj_scene_get_lights")
        cam = np.array(info.camera[:], F32)
    finally:
        lib.dipl_obj_scene_destroy(h)
    materials = [Material(name=bytes(names[i]).split(b"\0", 1)[0].decode(errors="replace"),
                          ambient=mvals[i, 0:3].copy(), diffuse=mvals[i, 3:6].copy(), specular=mvals[i, 6:9].copy(),
                          transmittance=mvals[i, 9:12].copy(), emission=mvals[i, 12:15].copy(),
                          shininess=mvals[i, 15], ior=mvals[i, 16], r_ior=mvals[i, 17], dissolve=mvals[i, 18])
                 for i in range(nm)]
    area = [AreaLight(color=al_color[i].copy(), triangle_id=int(al_id[i]), surface_area=al_area[i]) for i in range(na)]
    points = [PointLight(pos=pls[i, 0:3].copy(), color=pls[i, 3:6].copy(), power=pls[i, 6]) for i in range(npl)]
    camera = Camera(pos=cam[0:3].copy(), dir=cam[3:6].copy(), up=cam[6:9].copy(), fov=cam[9], far=cam[10])
    return Scene(positions=pos, normals=nrm, has_vertex_normals=has_n.astype(bool), geom_normals=geom,
                 material_ids=mat, materials=materials, area_lights=area, point_lights=points, camera=camera)


def render_scene_frame(scene: Scene, width: int, height: int, seed: int = 1, config=None, stats=None):
    """One wavefront frame of an OBJ scene on the device: upload SoA vertices, PLOC build, pinhole primary rays
    from the scene camera, closest hits, cosine bounce rays, closest hits. Returns (bvh, frame dict)."""
    import torch

    from . import accel
    bvh = accel.GpuPlocBvh()
    bvh.Build(config or accel.AccelerationStructureConfig(), stats if stats is not None else accel.Stats(),
              torch.from_numpy(scene.triangles()).cuda())
    return bvh, accel.trace_frame(bvh, scene.camera.as_dict(), width, height, seed, stats=stats)
