"""Seeded synthetic meshes and ray batches for the BVH build-and-trace workloads.

Every random number comes from the counter-based avalanche hash the reference
uses for its own sampling (``HashU32`` / ``U01FromU32``, src/util/util.h:24-37),
so a (seed, stream, index) triple always maps to the same value on any machine.
Normals and log-normals use Box-Muller on two such uniforms.

Triangles are returned as a float32 array of shape (N, 3, 3): triangle, corner
(v0, v1, v2), xyz. That is the per-triangle corner order of the reference's
``Triangle{Vertex v0, v1, v2}`` (src/scene/triangle.h:12-16) and of the SoA
``tri_v{0,1,2}_pos`` arrays its GPU scene uploads (src/gpu/scene/gpu_scene.h:18-20).

Rays are float32 (R, 8): origin xyz, tmin, direction xyz, tmax. ``tmin`` is the
reference's hit threshold ``kEpsilon`` = 1e-6 (src/util/util.h:15,
src/acceleration/sbvh.cc:85); ``tmax`` plays the role of ``Ray::t_max``
(src/scene/ray.h:7-11).

The workloads:

* ``small_scene``       — 5 axis-aligned unit quads (open box, 10 triangles) plus a
                          64x32 UV sphere (3968 triangles, radius 0.25, jittered centre);
                          512x512 pinhole primary rays + one cosine bounce per hit.
* ``displaced_sphere``  — 1024x512 UV sphere (1,046,528 triangles), radius 1 with a
                          4-octave value-noise displacement of amplitude 0.05; rays from
                          a radius-3 sphere into the inward hemisphere.
* ``soup``              — 16M triangles: centroids U[0,1]^3, edge lengths log-normal
                          (mu=-6, sigma=1.5), 20% skinny (1:50), random orientation;
                          random rays inside the unit cube.
* ``batched_meshes``    — 256 displaced spheres, triangle counts log-uniform in [1k, 2M].
* ``diff_scene``        — 256x128 displaced sphere (65,024 triangles) seen by a
                          1024x1024 pinhole camera, with a seeded target depth map.
"""
from __future__ import annotations

import math
import os

import numpy as np

K_EPSILON = np.float32(1e-6)          # reference kEpsilon (src/util/util.h:15)
K_INFINITY = np.float32(np.finfo(np.float32).max)  # reference kInfinity (util.h:16)

# Streams keep independent uses of one seed apart.
_S_JITTER, _S_NOISE, _S_RAY_O, _S_RAY_D, _S_SOUP, _S_BOUNCE, _S_BATCH, _S_TARGET = range(1, 9)


def hash_u32(x):
    """Avalanche hash, the reference's ``HashU32`` (src/util/util.h:24-32), on uint32 arrays."""
    x = np.asarray(x, dtype=np.uint32).copy()
    with np.errstate(over="ignore"):
        x ^= x >> np.uint32(16)
        x *= np.uint32(0x7FEB352D)
        x ^= x >> np.uint32(15)
        x *= np.uint32(0x846CA68B)
        x ^= x >> np.uint32(16)
    return x


def u01(x):
    """Top 24 bits to [0, 1): the reference's ``U01FromU32`` (src/util/util.h:34-37)."""
    return (np.asarray(x, dtype=np.uint32) >> np.uint32(8)).astype(np.float64) * (1.0 / 16777216.0)


def _key(seed, stream, idx, dim):
    """Mix (seed, stream, element index, dimension) into one uint32 key, then hash it."""
    idx = np.asarray(idx, dtype=np.uint64)
    with np.errstate(over="ignore"):
        k = (np.uint64(seed) * np.uint64(0x9E3779B1) + np.uint64(stream) * np.uint64(0x85EBCA6B)
             + np.uint64(dim) * np.uint64(0xC2B2AE35)) & np.uint64(0xFFFFFFFF)
        lo = (idx & np.uint64(0xFFFFFFFF)).astype(np.uint32)
        hi = (idx >> np.uint64(32)).astype(np.uint32)
        h = hash_u32(np.uint32(k) ^ hash_u32(lo ^ hash_u32(hi + np.uint32(dim))))
    return h


def rand01(seed, stream, idx, dim):
    """Uniform [0, 1) float64 per index."""
    return u01(_key(seed, stream, idx, dim))


def randn(seed, stream, idx, dim):
    """Standard normal per index (Box-Muller on dims 2*dim, 2*dim+1)."""
    u1 = rand01(seed, stream, idx, 2 * dim)
    u2 = rand01(seed, stream, idx, 2 * dim + 1)
    u1 = np.maximum(u1, 1.0 / 16777216.0)
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)


# ---------------------------------------------------------------------------------------------
# Value noise
# ---------------------------------------------------------------------------------------------

def _lattice(seed, ix, iy, iz, octave):
    with np.errstate(over="ignore"):
        k = (ix.astype(np.int64) * 73856093) ^ (iy.astype(np.int64) * 19349663) ^ (iz.astype(np.int64) * 83492791)
        k = (k & 0xFFFFFFFF).astype(np.uint32)
        h = hash_u32(k ^ hash_u32(np.uint32((seed * 2654435761 + octave * 40503 + _S_NOISE) & 0xFFFFFFFF)))
    return u01(h) * 2.0 - 1.0


def value_noise(p, seed, octaves=4, base_freq=4.0):
    """4-octave value noise in [-1, 1] at float64 points p (..., 3); smoothstep-interpolated lattice."""
    total = np.zeros(p.shape[:-1])
    amp, norm, freq = 1.0, 0.0, base_freq
    for o in range(octaves):
        q = p * freq
        i0 = np.floor(q)
        f = q - i0
        w = f * f * (3.0 - 2.0 * f)
        i0 = i0.astype(np.int64)
        acc = np.zeros(p.shape[:-1])
        for dx in (0, 1):
            wx = w[..., 0] if dx else 1.0 - w[..., 0]
            for dy in (0, 1):
                wy = w[..., 1] if dy else 1.0 - w[..., 1]
                for dz in (0, 1):
                    wz = w[..., 2] if dz else 1.0 - w[..., 2]
                    acc += wx * wy * wz * _lattice(seed, i0[..., 0] + dx, i0[..., 1] + dy, i0[..., 2] + dz, o)
        total += amp * acc
        norm += amp
        amp *= 0.5
        freq *= 2.0
    return total / norm


# ---------------------------------------------------------------------------------------------
# Meshes
# ---------------------------------------------------------------------------------------------

def uv_sphere_indexed(nu, nv, radius=1.0, center=(0.0, 0.0, 0.0), displacement=0.0, seed=0):
    """UV sphere with ``nu`` longitude segments and ``nv`` latitude rings, pole fans included.

    Returns (vertices float64 (V,3), indices int64 (T,3)); T = 2*nu*(nv-1).
    ``displacement`` scales the radius by (1 + displacement * noise(direction)).
    """
    nu, nv = int(nu), int(nv)
    theta = np.arange(1, nv) * (np.pi / nv)                  # ring polar angles
    phi = np.arange(nu) * (2.0 * np.pi / nu)
    st, ct = np.sin(theta)[:, None], np.cos(theta)[:, None]
    ring = np.stack([st * np.cos(phi)[None, :], ct * np.ones((1, nu)), st * np.sin(phi)[None, :]], axis=-1)
    dirs = np.concatenate([np.array([[0.0, 1.0, 0.0]]), ring.reshape(-1, 3), np.array([[0.0, -1.0, 0.0]])])
    r = np.full(len(dirs), float(radius))
    if displacement:
        r = r * (1.0 + displacement * value_noise(dirs, seed))
    verts = dirs * r[:, None] + np.asarray(center, dtype=np.float64)[None, :]
    top, bot = 0, len(dirs) - 1

    def vid(ring_i, seg):
        return 1 + ring_i * nu + (seg % nu)

    seg = np.arange(nu)
    tris = [np.stack([np.full(nu, top), vid(0, seg + 1), vid(0, seg)], axis=1)]
    for k in range(nv - 2):
        a, b = vid(k, seg), vid(k, seg + 1)
        c, d = vid(k + 1, seg), vid(k + 1, seg + 1)
        tris.append(np.stack([a, b, d], axis=1))
        tris.append(np.stack([a, d, c], axis=1))
    tris.append(np.stack([np.full(nu, bot), vid(nv - 2, seg), vid(nv - 2, seg + 1)], axis=1))
    idx = np.concatenate(tris).astype(np.int64)
    # interleave the quad halves so triangle order follows the surface ring by ring
    return verts, idx


def uv_sphere(nu, nv, radius=1.0, center=(0.0, 0.0, 0.0), displacement=0.0, seed=0):
    """Triangle soup (N, 3, 3) float32 of ``uv_sphere_indexed``."""
    v, i = uv_sphere_indexed(nu, nv, radius, center, displacement, seed)
    return v[i].astype(np.float32)


def open_box():
    """Five axis-aligned unit quads (10 triangles): floor, ceiling, back, left and right walls of [-0.5, 0.5]^3."""
    h = 0.5
    quads = [
        [(-h, -h, -h), (h, -h, -h), (h, -h, h), (-h, -h, h)],    # floor   y=-0.5
        [(-h, h, -h), (-h, h, h), (h, h, h), (h, h, -h)],        # ceiling y=+0.5
        [(-h, -h, -h), (-h, h, -h), (h, h, -h), (h, -h, -h)],    # back    z=-0.5
        [(-h, -h, -h), (-h, -h, h), (-h, h, h), (-h, h, -h)],    # left    x=-0.5
        [(h, -h, -h), (h, h, -h), (h, h, h), (h, -h, h)],        # right   x=+0.5
    ]
    tris = []
    for a, b, c, d in quads:
        tris.append([a, b, c])
        tris.append([a, c, d])
    return np.asarray(tris, dtype=np.float32)


# ---------------------------------------------------------------------------------------------
# Rays
# ---------------------------------------------------------------------------------------------

def _normalize(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def pack_rays(o, d, tmin=K_EPSILON, tmax=K_INFINITY):
    n = len(o)
    r = np.empty((n, 8), dtype=np.float32)
    r[:, 0:3] = o
    r[:, 3] = tmin
    r[:, 4:7] = d
    r[:, 7] = tmax
    return r


def pinhole_rays(width, height, cam_pos, cam_dir, cam_up, fov, far):
    """Primary rays, one per pixel, row-major from the top-left pixel.

    The camera basis follows the reference's CPU and GPU renderers
    (src/renderer/cpu_raytracer.cc:64-73, src/renderer/gpu_renderer.cc:25-35): right = normalize(dir x up),
    gw = 2 tan(fov/2), gh = gw*h/w, qw = right*gw/(w-1), qh = -up*gh/(h-1),
    p00 = dir - right*gw/2 + up*gh/2, ray dir = normalize(p00 + qw*x + qh*y), t_max = far.
    Evaluated in float32 like the reference.
    """
    f = np.float32
    cam_dir = np.asarray(cam_dir, f)
    cam_up = np.asarray(cam_up, f)
    right = np.cross(cam_dir, cam_up).astype(f)
    right = (right / np.sqrt((right * right).sum())).astype(f)
    gw = f(2.0 * math.tan(f(fov) / f(2.0)))
    gh = f(gw * (f(height) / f(width)))
    qw = right * f(gw / f(width - 1))
    qh = -cam_up * f(gh / f(height - 1))
    p00 = cam_dir - right * f(gw / f(2)) + cam_up * f(gh / f(2))
    ys, xs = np.meshgrid(np.arange(height, dtype=f), np.arange(width, dtype=f), indexing="ij")
    d = p00[None, :] + qw[None, :] * xs.reshape(-1, 1) + qh[None, :] * ys.reshape(-1, 1)
    d = (d / np.sqrt((d * d).sum(axis=1, keepdims=True))).astype(f)
    o = np.broadcast_to(np.asarray(cam_pos, f), d.shape)
    return pack_rays(o, d, K_EPSILON, f(far))


def sphere_inward_rays(n, seed, radius=3.0):
    """Origins uniform on a sphere of ``radius``; directions uniform over the inward hemisphere."""
    idx = np.arange(n, dtype=np.uint64)
    z = 1.0 - 2.0 * rand01(seed, _S_RAY_O, idx, 0)
    a = 2.0 * np.pi * rand01(seed, _S_RAY_O, idx, 1)
    s = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    p = np.stack([s * np.cos(a), s * np.sin(a), z], axis=1)
    o = p * radius
    z2 = 1.0 - 2.0 * rand01(seed, _S_RAY_D, idx, 0)
    a2 = 2.0 * np.pi * rand01(seed, _S_RAY_D, idx, 1)
    s2 = np.sqrt(np.maximum(0.0, 1.0 - z2 * z2))
    d = np.stack([s2 * np.cos(a2), s2 * np.sin(a2), z2], axis=1)
    flip = (d * p).sum(axis=1) > 0.0
    d[flip] = -d[flip]
    return pack_rays(o.astype(np.float32), d.astype(np.float32))


def random_rays(n, seed, lo=0.0, hi=1.0):
    """Origins uniform in [lo, hi]^3, directions uniform on the sphere, t_max = kInfinity."""
    return _by_index_ranges(n, lambda a, b: _random_rays_range(a, b, seed, lo, hi), (8,), np.float32)


def _random_rays_range(first, last, seed, lo, hi):
    idx = np.arange(first, last, dtype=np.uint64)
    o = lo + (hi - lo) * np.stack([rand01(seed, _S_RAY_O, idx, k) for k in range(3)], axis=1)
    z = 1.0 - 2.0 * rand01(seed, _S_RAY_D, idx, 0)
    a = 2.0 * np.pi * rand01(seed, _S_RAY_D, idx, 1)
    s = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    d = np.stack([s * np.cos(a), s * np.sin(a), z], axis=1)
    return pack_rays(o.astype(np.float32), d.astype(np.float32))


def ray_epsilon(pos, t):
    """Self-intersection offset of a hit point: the reference's ``RayEpsilon`` (src/scene/ray.h:15-24)."""
    f = np.float32
    p_scale = np.maximum(np.abs(pos).max(axis=1), f(1.0))
    t_scale = np.maximum(t, f(1.0))
    bias = np.maximum(f(1e-6) * p_scale, f(1e-7) * t_scale)
    return np.clip(bias, f(1e-7), f(1e-3)).astype(f)


def bounce_rays(tris, rays, prim, t, seed):
    """One cosine-weighted bounce ray per primary hit (misses get a zero-length, never-hitting ray).

    The origin is the hit point offset by ``ray_epsilon`` along the geometric normal on the side
    of the new direction, like the reference's ``OffsetRayOrigin`` (src/renderer/cpu_raytracer.cc:40-45).
    Returns (bounce rays (R, 8), mask of rays that carry a real bounce).
    """
    f = np.float32
    n = len(rays)
    hit = prim >= 0
    out = pack_rays(np.zeros((n, 3), f), np.tile(np.array([0, 0, 1], f), (n, 1)), K_EPSILON, f(0.0))
    if not hit.any():
        return out, hit
    hi = np.nonzero(hit)[0]
    tri = tris[prim[hi]].astype(np.float64)
    ng = _normalize(np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0]))
    d_in = rays[hi, 4:7].astype(np.float64)
    facing = (ng * d_in).sum(axis=1) > 0.0
    ng[facing] = -ng[facing]                      # normal facing the incoming ray
    u1 = rand01(seed, _S_BOUNCE, hi.astype(np.uint64), 0)
    u2 = rand01(seed, _S_BOUNCE, hi.astype(np.uint64), 1)
    r = np.sqrt(u1)
    a = 2.0 * np.pi * u2
    lx, ly, lz = r * np.cos(a), r * np.sin(a), np.sqrt(np.maximum(0.0, 1.0 - u1))
    helper = np.where(np.abs(ng[:, :1]) > 0.9, np.array([[0.0, 1.0, 0.0]]), np.array([[1.0, 0.0, 0.0]]))
    tx = _normalize(np.cross(helper, ng))
    ty = np.cross(ng, tx)
    d = _normalize(lx[:, None] * tx + ly[:, None] * ty + lz[:, None] * ng).astype(f)
    pos = (rays[hi, 0:3] + rays[hi, 4:7] * t[hi, None]).astype(f)
    eps = ray_epsilon(pos, t[hi].astype(f))
    o = (pos + ng.astype(f) * eps[:, None]).astype(f)
    out[hi, 0:3] = o
    out[hi, 4:7] = d
    out[hi, 7] = K_INFINITY
    return out, hit


# ---------------------------------------------------------------------------------------------
# Workloads
# ---------------------------------------------------------------------------------------------

SMALL_CAMERA = dict(cam_pos=(0.0, 0.0, 1.6), cam_dir=(0.0, 0.0, -1.0), cam_up=(0.0, 1.0, 0.0), fov=0.9, far=100.0)


def small_scene(seed=1, width=512, height=512, sphere_nu=64, sphere_nv=32):
    """Open box (10 triangles) + 64x32 UV sphere (radius 0.25, centre jittered by the seed); primary rays."""
    idx = np.arange(3, dtype=np.uint64)
    jitter = (rand01(seed, _S_JITTER, idx, 0) - 0.5) * 0.3
    center = np.array([0.0, -0.2, -0.1]) + jitter
    tris = np.concatenate([open_box(), uv_sphere(sphere_nu, sphere_nv, 0.25, center)])
    rays = pinhole_rays(width, height, **SMALL_CAMERA)
    return tris, rays


def displaced_sphere(seed=2, nu=1024, nv=512, n_rays=4 * 1024 * 1024):
    """1024x512 displaced unit sphere (amplitude 0.05) and rays from the radius-3 sphere inward."""
    tris = uv_sphere(nu, nv, 1.0, (0.0, 0.0, 0.0), displacement=0.05, seed=seed)
    rays = sphere_inward_rays(n_rays, seed)
    return tris, rays


def _by_index_ranges(n, make, shape, dtype, threads=None, chunk=1 << 20):
    """Fills an (n, *shape) array with make(lo, hi) over index ranges on host threads. Generators whose records
    depend only on their index give the same array for any split; numpy releases the interpreter lock inside its
    loops, so large workloads are made in parallel."""
    if n <= chunk:
        return make(0, n)
    from concurrent.futures import ThreadPoolExecutor
    out = np.empty((n, *shape), dtype)

    def part(lo):
        out[lo:min(n, lo + chunk)] = make(lo, min(n, lo + chunk))

    with ThreadPoolExecutor(max_workers=threads or min(32, os.cpu_count() or 1)) as ex:
        list(ex.map(part, range(0, n, chunk)))
    return out


def soup(n, seed=3, skinny_frac=0.2, mu=-6.0, sigma=1.5, threads=None):
    """Triangle soup: centroids U[0,1]^3, log-normal edge lengths, ``skinny_frac`` of 1:50 aspect, random rotation.
    Triangle i depends only on i, so ``soup(n)[:k]`` equals ``soup(k)``."""
    return _by_index_ranges(n, lambda lo, hi: _soup_range(lo, hi, seed, skinny_frac, mu, sigma), (3, 3),
                            np.float32, threads)


def _soup_range(lo, hi, seed, skinny_frac, mu, sigma):
    n = hi - lo
    idx = np.arange(lo, hi, dtype=np.uint64)
    c = np.stack([rand01(seed, _S_SOUP, idx, k) for k in range(3)], axis=1)
    ell = np.exp(mu + sigma * randn(seed, _S_SOUP, idx, 3))
    skinny = rand01(seed, _S_SOUP, idx, 8) < skinny_frac
    ell_b = np.where(skinny, ell / 50.0, ell)
    phi = np.deg2rad(30.0 + 120.0 * rand01(seed, _S_SOUP, idx, 9))
    p0 = np.zeros((n, 3))
    p1 = np.stack([ell, np.zeros(n), np.zeros(n)], axis=1)
    p2 = np.stack([ell_b * np.cos(phi), ell_b * np.sin(phi), np.zeros(n)], axis=1)
    # uniform random rotation from a normalised 4-D Gaussian (a random unit quaternion)
    q = np.stack([randn(seed, _S_SOUP, idx, 10 + k) for k in range(4)], axis=1)
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    rot = np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], axis=1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], axis=1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], axis=1),
    ], axis=1)
    pts = np.stack([p0, p1, p2], axis=1)
    pts = pts - pts.mean(axis=1, keepdims=True)
    pts = np.einsum("nij,nkj->nki", rot, pts) + c[:, None, :]
    return pts.astype(np.float32)


def batched_mesh_sizes(count=256, seed=4, lo=1000, hi=2_000_000):
    """Per-mesh (nu, nv) with 2*nu*(nv-1) close to a log-uniform target in [lo, hi], nu = 2*nv."""
    idx = np.arange(count, dtype=np.uint64)
    target = np.exp(np.log(lo) + (np.log(hi) - np.log(lo)) * rand01(seed, _S_BATCH, idx, 0))
    sizes = []
    for tg in target:
        nv = max(3, int(round(math.sqrt(tg / 4.0 + 0.25) + 0.5)))
        sizes.append((2 * nv, nv))
    return sizes


def batched_meshes(count=256, seed=4, lo=1000, hi=2_000_000):
    """``count`` independent noise-displaced spheres; returns a list of (N_i, 3, 3) float32 arrays."""
    out = []
    for m, (nu, nv) in enumerate(batched_mesh_sizes(count, seed, lo, hi)):
        out.append(uv_sphere(nu, nv, 1.0, (0.0, 0.0, 0.0), displacement=0.05, seed=seed * 1000 + m))
    return out


DIFF_CAMERA = dict(cam_pos=(0.0, 0.0, 3.0), cam_dir=(0.0, 0.0, -1.0), cam_up=(0.0, 1.0, 0.0), fov=0.8, far=100.0)


def diff_scene(seed=5, nu=256, nv=128, width=1024, height=1024):
    """65k-triangle displaced sphere (indexed), pinhole rays, and the displacement seed of the target."""
    verts, idx = uv_sphere_indexed(nu, nv, 1.0, (0.0, 0.0, 0.0), displacement=0.05, seed=seed)
    rays = pinhole_rays(width, height, **DIFF_CAMERA)
    return verts, idx, rays
