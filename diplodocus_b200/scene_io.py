"""OBJ scene path into the engine: the reference's ObjSceneLoader, restated on the host, feeding device SoA.

Replaces ``ObjSceneLoader::Load / LoadObj / LoadMetadata`` (src/io/scene/obj_scene_loader.cc:20-205) and the
parts of its vendored tinyobjloader 2.0 (third-party/tinyobjloader/tiny_obj_loader.h) that decide which
triangles come out: index fix-up (1-based, negative = relative to the vertices read so far), the split of a quad
along its shorter diagonal (exportGroupsToShape), ear clipping of larger polygons, ``usemtl`` / ``mtllib``
resolution and the MTL keys the reference reads. Triangles come out in file order, positions and normals bit
for bit as the reference's float32 parse gives them; the geometric normal and the area of emissive triangles
are evaluated in float32 in the reference's operation order (scene.cc:18-21, triangle.h:22-34), so area lights
match it exactly.

``Scene.device_vertices`` gives the three SoA vertex arrays that ``dipl_build_desc`` takes, so a Cornell scene
runs file -> PLOC build -> trace through the engine (``render_scene_frame``).

Deliberate differences: a vertex or normal index out of range fails the load (the reference reads out of
bounds); a ``.meta`` value must be a complete number token (the reference's stream extraction would accept a
numeric prefix).
"""
from __future__ import annotations

import logging
import os
import re
from dataclasses import dataclass, field

import numpy as np

log = logging.getLogger(__name__)

F32 = np.float32
_EPS = F32(1e-6)          # kEpsilon (src/util/util.h:15), Normalize's threshold
_FLT_EPS = F32(np.finfo(np.float32).eps)
_NUM_PREFIX = re.compile(r"[+-]?(\d+(\.\d*)?|\.\d+)([eE][+-]?\d+)?")
_NAN_INF = re.compile(r"[+-]?(nan|inf(inity)?)", re.IGNORECASE)
_NUM_FULL = re.compile(r"^[+-]?((\d+\.?\d*)|(\.\d+))([eE][+-]?\d+)?$")


def _num(tok: str) -> F32:
    """A number token of an OBJ or MTL file as tinyobj's tryParseDouble reads it: the longest decimal prefix
    (``-0.2200.`` is -0.22), or a nan / inf literal; string -> double -> float, like its static_cast."""
    m = _NAN_INF.match(tok)
    if m:
        return F32(float(m.group(0)))
    m = _NUM_PREFIX.match(tok)
    if not m:
        raise ValueError(f"expected number, got {tok!r}")
    val = float(m.group(0))
    if np.isinf(val):
        raise ValueError(f"number out of range: {tok!r}")
    return F32(val)


def _meta_num(tok: str) -> F32:
    """A .meta value: one complete decimal token."""
    if not _NUM_FULL.match(tok):
        raise ValueError(f"expected number, got {tok!r}")
    return F32(float(tok))


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
# Float32 geometry in the reference's operation order
# ---------------------------------------------------------------------------------------------------------
def _cross(a, b):
    # Cross (src/util/vec3.h:119-121)
    return np.array([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]], F32)


def _length(v) -> F32:
    # Length (vec3.h:109): sqrt((x*x + y*y) + z*z) in float
    return F32(np.sqrt(F32(F32(v[0] * v[0] + v[1] * v[1]) + v[2] * v[2])))


def _geom_normal(p0, p1, p2):
    # RecomputeTriangleGeometricNormal (triangle.h:22-26): Normalize(Cross(v1 - v0, v2 - v0)), zero if |c| <= 1e-6
    c = _cross(p1 - p0, p2 - p0)
    ln = _length(c)
    if ln <= _EPS:
        return np.zeros(3, F32)
    return (c / ln).astype(F32)


def _surface_area(p0, p1, p2) -> F32:
    # CalculateTriangleSurfaceArea (triangle.h:28-34): 0.5 * Length(Cross(v1 - v0, v2 - v0)), double then float
    return F32(0.5 * float(_length(_cross(p1 - p0, p2 - p0))))


# ---------------------------------------------------------------------------------------------------------
# Polygon triangulation (tinyobjloader exportGroupsToShape, triangulate = true, no mapbox earcut)
# ---------------------------------------------------------------------------------------------------------
def _pnpoly(vx, vy, tx, ty) -> bool:
    # Franklin's crossing test on the candidate ear, float arithmetic
    c = False
    j = 2
    for i in range(3):
        if (vy[i] > ty) != (vy[j] > ty):
            x = F32(F32(F32(vx[j] - vx[i]) * F32(ty - vy[i])) / F32(vy[j] - vy[i])) + vx[i]
            if tx < x:
                c = not c
        j = i
    return c


def _triangulate(face, v):
    """Triangles (as index triples into ``face``'s entries) tinyobj makes of one polygon face.

    ``face`` is a list of (v, vt, vn) index triples, ``v`` the (M, 3) float32 positions read so far.
    """
    n = len(face)
    nv = len(v)
    if n < 3:
        return []  # "Degenerated face": skipped
    if n == 3:
        return [(0, 1, 2)]
    if n == 4:
        if any(f[0] < 0 or f[0] >= nv for f in face):
            return []  # "Face with invalid vertex index": skipped
        p = [v[f[0]] for f in face]
        e02 = p[2] - p[0]
        e13 = p[3] - p[1]
        sqr02 = F32(F32(e02[0] * e02[0] + e02[1] * e02[1]) + e02[2] * e02[2])
        sqr13 = F32(F32(e13[0] * e13[0] + e13[1] * e13[1]) + e13[2] * e13[2])
        if sqr02 < sqr13:
            return [(0, 1, 2), (0, 2, 3)]
        return [(0, 1, 3), (1, 2, 3)]

    def pos(k):
        vi = face[k][0]
        return v[vi] if 0 <= vi < nv else None

    # projection plane: the first corner whose edge cross product has a component above FLT_EPSILON
    axes = [1, 2]
    for k in range(n):
        a, b, c = pos(k % n), pos((k + 1) % n), pos((k + 2) % n)
        if a is None or b is None or c is None:
            continue
        e0, e1 = b - a, c - b
        cx = abs(F32(e0[1] * e1[2] - e0[2] * e1[1]))
        cy = abs(F32(e0[2] * e1[0] - e0[0] * e1[2]))
        cz = abs(F32(e0[0] * e1[1] - e0[1] * e1[0]))
        if cx > _FLT_EPS or cy > _FLT_EPS or cz > _FLT_EPS:
            if not (cx > cy and cx > cz):
                axes[0] = 0
                if cz > cx and cz > cy:
                    axes[1] = 1
            break

    def proj(k):
        p = pos(k)
        if p is None:
            return F32(0.0), F32(0.0)
        return p[axes[0]], p[axes[1]]

    out = []
    remaining = list(range(n))  # positions in `face`
    guess = 0
    iterations = n
    previous = n
    while len(remaining) > 3 and iterations > 0:
        m = len(remaining)
        if guess >= m:
            guess -= m
        if previous != m:
            previous = m
            iterations = m
        else:
            iterations -= 1
        ind = [remaining[(guess + k) % m] for k in range(3)]
        vx, vy = zip(*(proj(k) for k in ind))
        e0x, e0y = F32(vx[1] - vx[0]), F32(vy[1] - vy[0])
        e1x, e1y = F32(vx[2] - vx[1]), F32(vy[2] - vy[1])
        cross = F32(F32(e0x * e1y) - F32(e0y * e1x))
        area = F32(F32(F32(vx[0] * vy[1]) - F32(vy[0] * vx[1])) * F32(0.5))
        if F32(cross * area) < F32(0.0):
            guess += 1
            continue
        overlap = False
        for other in range(3, m):
            p = pos(remaining[(guess + other) % m])
            if p is None:
                continue
            if _pnpoly(vx, vy, p[axes[0]], p[axes[1]]):
                overlap = True
                break
        if overlap:
            guess += 1
            continue
        out.append(tuple(ind))
        del remaining[(guess + 1) % m]
    if len(remaining) == 3:
        out.append(tuple(remaining))
    return out


# ---------------------------------------------------------------------------------------------------------
# MTL (tinyobjloader LoadMtlInternal: the keys the reference's Material keeps)
# ---------------------------------------------------------------------------------------------------------
def _new_material_values():
    z = lambda: np.zeros(3, F32)  # noqa: E731
    return {"name": "", "ambient": z(), "diffuse": z(), "specular": z(), "transmittance": z(), "emission": z(),
            "shininess": F32(1.0), "ior": F32(1.0), "dissolve": F32(1.0), "has_d": False, "has_tr": False,
            "has_kd": False}


def _load_mtl(path, materials, material_map) -> bool:
    """Appends the materials of one MTL file; False if it cannot be read or has a malformed number (materials
    completed before the error stay, as in tinyobj)."""
    try:
        with open(path, "r", encoding="utf-8", errors="replace") as f:
            lines = f.read().splitlines()
    except OSError:
        return False
    cur = _new_material_values()

    def flush():
        if cur["name"]:
            material_map.setdefault(cur["name"], len(materials))  # std::map::insert keeps the first
            materials.append(dict(cur))

    def rgb(toks):
        vals = [F32(0.0)] * 3
        for i in range(3):
            if i < len(toks):
                vals[i] = _num(toks[i])
        return np.array(vals, F32)

    try:
        for raw in lines:
            line = raw.lstrip("﻿").strip()
            if not line or line.startswith("#"):
                continue
            key, *toks = line.split()
            if key == "newmtl":
                flush()
                cur = _new_material_values()
                cur["name"] = toks[0] if toks else ""
            elif key == "Ka":
                cur["ambient"] = rgb(toks)
            elif key == "Kd":
                cur["diffuse"] = rgb(toks)
                cur["has_kd"] = True
            elif key == "Ks":
                cur["specular"] = rgb(toks)
            elif key in ("Kt", "Tf"):
                cur["transmittance"] = rgb(toks)
            elif key == "Ke":
                cur["emission"] = rgb(toks)
            elif key == "Ni":
                cur["ior"] = _num(toks[0]) if toks else F32(0.0)
            elif key == "Ns":
                cur["shininess"] = _num(toks[0]) if toks else F32(0.0)
            elif key == "d":
                cur["dissolve"] = _num(toks[0]) if toks else F32(0.0)
                cur["has_d"] = True
            elif key == "Tr":
                if not cur["has_d"]:
                    cur["dissolve"] = F32(F32(1.0) - (_num(toks[0]) if toks else F32(0.0)))
                cur["has_tr"] = True
            elif key == "map_Kd":
                if not cur["has_kd"]:
                    cur["diffuse"] = np.array([0.6, 0.6, 0.6], F32)
            # illum, textures and PBR keys do not reach the reference's Material
    except ValueError as e:
        log.error("ObjSceneLoader: %s: %s", path, e)
        return False
    flush()
    return True


# ---------------------------------------------------------------------------------------------------------
# OBJ
# ---------------------------------------------------------------------------------------------------------
def _fix_index(tok: str, count: int) -> int:
    i = int(tok)
    if i > 0:
        return i - 1
    if i < 0:
        return count + i
    raise ValueError("zero index")


def _load_obj(path, meta_camera, meta_lights) -> Scene | None:
    try:
        with open(path, "r", encoding="utf-8", errors="replace") as f:
            lines = f.read().splitlines()
    except OSError:
        log.error("ObjSceneLoader: Error reading file %s", path)
        return None
    base = os.path.dirname(path)
    v: list = []
    vn: list = []
    nvt = 0
    materials: list = []
    material_map: dict = {}
    loaded_mtl: set = set()
    material = -1
    pending: list = []       # faces since the last flush: (face, material id)
    out_faces: list = []     # (3 (v, vt, vn) triples, material id) in output order
    varr = np.zeros((0, 3), F32)

    def flush():
        nonlocal pending, varr
        if not pending:
            return
        varr = np.array(v, F32).reshape(-1, 3)
        for face, mat in pending:
            for a, b, c in _triangulate(face, varr):
                out_faces.append(((face[a], face[b], face[c]), mat))
        pending = []

    try:
        for raw in lines:
            line = raw.strip()
            if not line or line.startswith("#"):
                continue
            if "#" in line:
                line = line[:line.index("#")].rstrip()
            key, *toks = line.split()
            if key == "v":
                xyz = [_num(t) for t in toks[:3]] + [F32(0.0)] * (3 - min(3, len(toks)))
                v.append(xyz)
            elif key == "vn":
                vn.append([_num(t) for t in toks[:3]] + [F32(0.0)] * (3 - min(3, len(toks))))
            elif key == "vt":
                nvt += 1
            elif key == "f":
                face = []
                for t in toks:
                    parts = t.split("/")
                    vi = _fix_index(parts[0], len(v))
                    ti = _fix_index(parts[1], nvt) if len(parts) > 1 and parts[1] else -1
                    ni = _fix_index(parts[2], len(vn)) if len(parts) > 2 and parts[2] else -1
                    face.append((vi, ti, ni))
                pending.append((face, material))
            elif key == "usemtl":
                new = material_map.get(toks[0] if toks else "", -1)
                if new < 0:
                    log.warning("material [ '%s' ] not found in .mtl", toks[0] if toks else "")
                if new != material:
                    flush()
                    material = new
            elif key == "mtllib":
                for name in toks:  # the first file that loads; files loaded before are skipped
                    if name in loaded_mtl:
                        continue
                    if _load_mtl(os.path.join(base, name), materials, material_map):
                        loaded_mtl.add(name)
                        break
            elif key in ("g", "o"):
                flush()
            # s, l, p, vp and unknown keys add no triangles
        flush()
    except (ValueError, IndexError) as e:
        log.error("ObjSceneLoader: Error reading file %s: %s", path, e)
        return None

    varr = np.array(v, F32).reshape(-1, 3)
    narr = np.array(vn, F32).reshape(-1, 3)
    n = len(out_faces)
    positions = np.zeros((n, 9), F32)
    normals = np.zeros((n, 9), F32)
    has_n = np.zeros(n, bool)
    geom = np.zeros((n, 3), F32)
    mats = np.full(n, -1, np.int32)
    area_lights = []
    for i, (tri, mat) in enumerate(out_faces):
        vis = [t[0] for t in tri]
        if any(x < 0 or x >= len(varr) for x in vis):
            log.error("ObjSceneLoader: vertex index out of range in %s", path)
            return None
        p = [varr[x] for x in vis]
        positions[i] = np.concatenate(p)
        nis = [t[2] for t in tri]
        if all(x >= 0 for x in nis):
            if any(x >= len(narr) for x in nis):
                log.error("ObjSceneLoader: normal index out of range in %s", path)
                return None
            normals[i] = np.concatenate([narr[x] for x in nis])
            has_n[i] = True
        geom[i] = _geom_normal(*p)
        mats[i] = mat
        if mat >= 0 and np.any(materials[mat]["emission"] != 0):
            area_lights.append(AreaLight(color=materials[mat]["emission"].copy(), triangle_id=i,
                                         surface_area=_surface_area(*p)))
    mlist = [Material(name=m["name"], ambient=m["ambient"], diffuse=m["diffuse"], specular=m["specular"],
                      transmittance=m["transmittance"], emission=m["emission"], shininess=m["shininess"],
                      ior=m["ior"], r_ior=F32(F32(1.0) / m["ior"]), dissolve=m["dissolve"]) for m in materials]
    return Scene(positions=positions, normals=normals, has_vertex_normals=has_n, geom_normals=geom,
                 material_ids=mats, materials=mlist, area_lights=area_lights, point_lights=meta_lights,
                 camera=meta_camera)


def _load_metadata(path):
    """LoadMetadata (obj_scene_loader.cc:120-187): camera and point lights; None on any error."""
    try:
        with open(path, "r", encoding="utf-8", errors="replace") as f:
            toks = f.read().split()
    except OSError:
        log.error("ObjSceneLoader: Error reading metadata file %s", path)
        return None
    cam = Camera()
    lights = []
    i = 0

    def take(k):
        nonlocal i
        if i + k > len(toks):
            raise ValueError("missing value")
        vals = [_meta_num(t) for t in toks[i:i + k]]
        i += k
        return vals

    try:
        while i < len(toks):
            tok = toks[i]
            i += 1
            if tok == "cam_pos":
                cam.pos = np.array(take(3), F32)
            elif tok == "cam_up":
                cam.up = np.array(take(3), F32)
            elif tok == "cam_dir":
                cam.dir = np.array(take(3), F32)
            elif tok == "cam_fov":
                cam.fov = take(1)[0]
            elif tok == "cam_far":
                cam.far = take(1)[0]
            elif tok == "point_light":
                pos, color, power = take(3), take(3), take(1)[0]
                lights.append(PointLight(pos=np.array(pos, F32), color=np.array(color, F32), power=power))
            else:
                log.error("ObjSceneLoader: Unrecognized metadata token '%s'", tok)
                return None
    except ValueError:
        log.error("ObjSceneLoader: malformed metadata in %s", path)
        return None
    return cam, lights


def load_obj_scene(dirpath, name) -> Scene | None:
    """ObjSceneLoader::Load (obj_scene_loader.cc:189-205): ``<dirpath>/<name>.meta`` then ``<name>.obj`` (MTL
    files named by ``mtllib`` are looked up beside the OBJ). None where the reference returns std::nullopt."""
    basepath = os.path.join(str(dirpath), str(name))
    meta = _load_metadata(basepath + ".meta")
    if meta is None:
        return None
    return _load_obj(basepath + ".obj", *meta)


def render_scene_frame(scene: Scene, width: int, height: int, seed: int = 1, config=None, stats=None):
    """One wavefront frame of an OBJ scene on the device: upload SoA vertices, PLOC build, pinhole primary rays
    from the scene camera, closest hits, cosine bounce rays, closest hits. Returns (bvh, frame dict)."""
    import torch

    from . import accel
    bvh = accel.GpuPlocBvh()
    bvh.Build(config or accel.AccelerationStructureConfig(), stats if stats is not None else accel.Stats(),
              torch.from_numpy(scene.triangles()).cuda())
    return bvh, accel.trace_frame(bvh, scene.camera.as_dict(), width, height, seed, stats=stats)
