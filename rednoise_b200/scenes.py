"""Seeded synthetic scenes of the path-tracing workloads (no dataset involved).

Every scene is generated from a 64-bit seed with splitmix64 (geometry and
material assignment), so any process reproduces the same triangles bit for bit.

* ``cornell_box()``  -- a 5.56 m axis-aligned room of 10 wall triangles (left wall
  albedo (0.63, 0.065, 0.05), right wall (0.14, 0.45, 0.091), others 0.725), two
  Lambertian boxes of 12 triangles (rotated +18 and -15 degrees) and a
  0.13 x 0.105 m emissive ceiling quad of radiance (17, 12, 4): 36 triangles.
* ``icosphere_scene()`` -- the room plus a level-8 icosphere (20 * 4^8 =
  1,310,720 triangles) of radius 1.2 m displaced along its normals by seeded
  4-octave value noise of amplitude 0.08 m; per-triangle materials by seeded
  hash: 60 % Lambert (albedo U[0.2, 0.8]^3), 25 % GGX (roughness U[0.05, 0.5]),
  15 % dielectric (IOR 1.5).
* ``soup_scene()`` -- the room plus a seeded random triangle soup.
* ``batch_jobs()`` -- the 64-job batched workload (soup sizes, resolutions, spp).
* ``views()`` -- seeded camera views for multi-view inverse rendering.

The pinhole camera looks down -z through the open front of the room with a
40 degree vertical field of view.
"""
from __future__ import annotations

import math
from typing import Dict

import numpy as np

LAMBERT, GGX, DIELECTRIC = 0, 1, 2
# reference Material enum values (framework/ModelTriangle.h:12-24)
REF_DIFFUSE, REF_GLASS, REF_METAL, REF_EMISSIVE = 0, 2, 6, 10

HALF = 2.78  # half the 5.56 m room
CAMERA_Z = HALF + HALF / math.tan(math.radians(20.0))

_MASK = (1 << 64) - 1


def splitmix64(x: np.ndarray) -> np.ndarray:
    """splitmix64 finaliser (Steele, Lea, Flood 2014) on uint64 arrays."""
    with np.errstate(over="ignore"):
        z = (x + np.uint64(0x9E3779B97F4A7C15)) & np.uint64(_MASK)
        z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & np.uint64(_MASK)
        z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & np.uint64(_MASK)
        return z ^ (z >> np.uint64(31))


def uniform(seed: int, stream: int, index: np.ndarray) -> np.ndarray:
    """Deterministic U[0, 1) doubles for (seed, stream, index)."""
    idx = np.asarray(index, dtype=np.uint64)
    with np.errstate(over="ignore"):
        key = np.uint64((seed * 0x100000001B3 + stream * 0x9E3779B1) & _MASK)
        h = splitmix64(splitmix64(idx ^ key) + np.uint64(stream))
    return (h >> np.uint64(11)).astype(np.float64) * (1.0 / float(1 << 53))


def camera(width: int, height: int, vfov_deg: float = 40.0) -> Dict:
    return {
        "position": (0.0, 0.0, CAMERA_Z),
        "target": (0.0, 0.0, 0.0),
        "up": (0.0, 1.0, 0.0),
        "vfov_deg": vfov_deg,
        "width": width,
        "height": height,
    }


def _quad(a, b, c, d):
    """Two triangles (a, b, c) and (a, c, d); counter-clockwise seen from the front."""
    return [np.array([a, b, c], np.float64), np.array([a, c, d], np.float64)]


def _box(center, size, angle_deg):
    """12 outward-facing triangles of a box rotated about +y."""
    hx, hy, hz = (s / 2.0 for s in size)
    ca, sa = math.cos(math.radians(angle_deg)), math.sin(math.radians(angle_deg))

    def p(x, y, z):
        return (center[0] + ca * x + sa * z, center[1] + y, center[2] - sa * x + ca * z)

    c = {(i, j, k): p(i * hx, j * hy, k * hz) for i in (-1, 1) for j in (-1, 1) for k in (-1, 1)}
    tris = []
    tris += _quad(c[(-1, 1, -1)], c[(-1, 1, 1)], c[(1, 1, 1)], c[(1, 1, -1)])  # top (+y)
    tris += _quad(c[(-1, -1, -1)], c[(1, -1, -1)], c[(1, -1, 1)], c[(-1, -1, 1)])  # bottom
    tris += _quad(c[(-1, -1, 1)], c[(1, -1, 1)], c[(1, 1, 1)], c[(-1, 1, 1)])  # +z
    tris += _quad(c[(1, -1, -1)], c[(-1, -1, -1)], c[(-1, 1, -1)], c[(1, 1, -1)])  # -z
    tris += _quad(c[(1, -1, 1)], c[(1, -1, -1)], c[(1, 1, -1)], c[(1, 1, 1)])  # +x
    tris += _quad(c[(-1, -1, -1)], c[(-1, -1, 1)], c[(-1, 1, 1)], c[(-1, 1, -1)])  # -x
    return tris


def _room(light_scale: float = 1.0):
    h = HALF
    walls, albedo = [], []
    grey = (0.725, 0.725, 0.725)
    for tris, col in (
        (_quad((-h, -h, h), (h, -h, h), (h, -h, -h), (-h, -h, -h)), grey),  # floor, normal +y
        (_quad((-h, h, -h), (h, h, -h), (h, h, h), (-h, h, h)), grey),  # ceiling, normal -y
        (_quad((-h, -h, -h), (h, -h, -h), (h, h, -h), (-h, h, -h)), grey),  # back wall, normal +z
        (_quad((-h, -h, h), (-h, -h, -h), (-h, h, -h), (-h, h, h)), (0.63, 0.065, 0.05)),  # left, +x
        (_quad((h, -h, -h), (h, -h, h), (h, h, h), (h, h, -h)), (0.14, 0.45, 0.091)),  # right, -x
    ):
        walls += tris
        albedo += [col, col]
    boxes = _box((0.95, -h + 0.825, 0.75), (1.65, 1.65, 1.65), -15.0) + _box(
        (-0.95, -h + 1.65, -0.9), (1.65, 3.30, 1.65), 18.0
    )
    albedo += [grey] * len(boxes)
    lw, ld = 0.13 / 2.0 * light_scale, 0.105 / 2.0 * light_scale
    y = h - 1e-3
    light = _quad((-lw, y, -ld), (lw, y, -ld), (lw, y, ld), (-lw, y, ld))  # normal -y (faces down)
    tris = walls + boxes + light
    v = np.stack([t.reshape(9) for t in tris]).astype(np.float32)
    n = v.shape[0]
    alb = np.zeros((n, 3), np.float32)
    alb[: len(albedo)] = np.asarray(albedo, np.float32)
    em = np.zeros((n, 3), np.float32)
    em[-2:] = (17.0, 12.0, 4.0)
    return v, alb, em


def _finish(v, albedo, emission, material, param) -> Dict:
    n = v.shape[0]
    ref_material = np.full(n, REF_DIFFUSE, np.int32)
    ref_material[material == GGX] = REF_METAL
    ref_material[material == DIELECTRIC] = REF_GLASS
    emissive = emission.max(axis=1) > 0
    ref_material[emissive] = REF_EMISSIVE
    ref_rgb = np.clip((albedo * 255.0).astype(np.int32), 0, 255)
    # Reference emission is colour/255*4: carry the emitter's chromaticity.
    if emissive.any():
        e = emission[emissive]
        ref_rgb[emissive] = np.clip((e / e.max(axis=1, keepdims=True) * 255.0).astype(np.int32), 0, 255)
    ref_rough = np.where(material == GGX, np.sqrt(np.maximum(param, 0.0)), 0.2).astype(np.float32)
    return {
        "vertices": np.ascontiguousarray(v, np.float32),
        "albedo": np.ascontiguousarray(albedo, np.float32),
        "emission": np.ascontiguousarray(emission, np.float32),
        "material": np.ascontiguousarray(material, np.int32),
        "material_param": np.ascontiguousarray(param, np.float32),
        "ref_rgb": ref_rgb,
        "ref_material": ref_material,
        "ref_roughness": ref_rough,
    }


def cornell_box(light_scale: float = 1.0) -> Dict:
    """The 36-triangle Cornell box (all Lambertian, one emitter quad).
    ``light_scale`` scales the light quad's sides (1 = the 0.13 x 0.105 m quad;
    statistical tests use 10 for a low-variance image)."""
    v, alb, em = _room(light_scale)
    n = v.shape[0]
    return _finish(v, alb, em, np.zeros(n, np.int32), np.full(n, 0.2, np.float32))


# ---- icosphere ------------------------------------------------------------------------

def _icosahedron():
    t = (1.0 + math.sqrt(5.0)) / 2.0
    verts = np.array(
        [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)], np.float64)
    verts /= np.linalg.norm(verts, axis=1, keepdims=True)
    faces = np.array(
        [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
         (6, 2, 10), (8, 6, 7), (9, 8, 1)], np.int64)
    return verts[faces]  # (20, 3, 3) outward CCW


def icosphere(level: int) -> np.ndarray:
    """(20 * 4^level, 3, 3) unit-sphere triangles; shared vertices are bit-identical."""
    tris = _icosahedron()
    for _ in range(level):
        a, b, c = tris[:, 0], tris[:, 1], tris[:, 2]

        def mid(p, q):
            m = p + q
            return m / np.sqrt((m * m).sum(axis=1, keepdims=True))

        ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
        tris = np.stack(
            [np.stack([a, ab, ca], 1), np.stack([ab, b, bc], 1), np.stack([ca, bc, c], 1),
             np.stack([ab, bc, ca], 1)], 1).reshape(-1, 3, 3)
    return tris


def value_noise(p: np.ndarray, seed: int, octaves: int = 4) -> np.ndarray:
    """Seeded fractal lattice value noise in [-1, 1] (smoothstep-trilinear, octave gain 0.5)."""
    total = np.zeros(p.shape[0])
    norm = 0.0
    amp, freq = 1.0, 1.5
    for o in range(octaves):
        q = p * freq
        i0 = np.floor(q).astype(np.int64)
        f = q - i0
        w = f * f * (3.0 - 2.0 * f)
        acc = np.zeros(p.shape[0])
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    key = ((i0[:, 0] + dx) * 73856093) ^ ((i0[:, 1] + dy) * 19349663) ^ ((i0[:, 2] + dz) * 83492791)
                    val = uniform(seed, 100 + o, key.astype(np.uint64)) * 2.0 - 1.0
                    wx = w[:, 0] if dx else 1.0 - w[:, 0]
                    wy = w[:, 1] if dy else 1.0 - w[:, 1]
                    wz = w[:, 2] if dz else 1.0 - w[:, 2]
                    acc += wx * wy * wz * val
        total += amp * acc
        norm += amp
        amp *= 0.5
        freq *= 2.0
    return total / norm


def icosphere_scene(level: int = 8, seed: int = 0x5EED0002, radius: float = 1.2, amplitude: float = 0.08,
                    center=(0.0, -1.45, 0.0)) -> Dict:
    """The room plus the displaced, material-mixed icosphere (level 8: 1,310,720 triangles)."""
    rv, ralb, rem = _room()
    sph = icosphere(level)  # unit sphere, float64
    flat = sph.reshape(-1, 3)
    disp = radius + amplitude * value_noise(flat * 2.0, seed)
    pts = flat * disp[:, None] + np.asarray(center)[None, :]
    sv = pts.reshape(-1, 9).astype(np.float32)
    m = sv.shape[0]
    idx = np.arange(m, dtype=np.uint64)
    u = uniform(seed, 1, idx)
    material = np.where(u < 0.60, LAMBERT, np.where(u < 0.85, GGX, DIELECTRIC)).astype(np.int32)
    albedo = (0.2 + 0.6 * np.stack([uniform(seed, 2 + k, idx) for k in range(3)], 1)).astype(np.float32)
    param = np.where(material == GGX, 0.05 + 0.45 * uniform(seed, 5, idx), 1.5).astype(np.float32)
    param[material == LAMBERT] = 0.2
    n0 = rv.shape[0]
    v = np.concatenate([rv, sv])
    alb = np.concatenate([ralb, albedo])
    em = np.concatenate([rem, np.zeros((m, 3), np.float32)])
    mat = np.concatenate([np.zeros(n0, np.int32), material])
    par = np.concatenate([np.full(n0, 0.2, np.float32), param])
    return _finish(v, alb, em, mat, par)


def soup_scene(count: int, seed: int) -> Dict:
    """The room plus ``count`` random triangles inside it (edges U[0.01, 0.2] m), all Lambertian."""
    rv, ralb, rem = _room()
    idx = np.arange(count, dtype=np.uint64)
    c = np.stack([uniform(seed, k, idx) for k in range(3)], 1) * (2 * HALF - 0.4) - (HALF - 0.2)
    verts = [c]
    for j in range(2):
        d = np.stack([uniform(seed, 10 + 4 * j + k, idx) * 2.0 - 1.0 for k in range(3)], 1)
        d /= np.maximum(np.linalg.norm(d, axis=1, keepdims=True), 1e-9)
        ln = 0.01 + 0.19 * uniform(seed, 20 + j, idx)
        verts.append(c + d * ln[:, None])
    sv = np.stack(verts, 1).reshape(-1, 9).astype(np.float32)
    albedo = (0.2 + 0.6 * np.stack([uniform(seed, 30 + k, idx) for k in range(3)], 1)).astype(np.float32)
    n0 = rv.shape[0]
    v = np.concatenate([rv, sv])
    alb = np.concatenate([ralb, albedo])
    em = np.concatenate([rem, np.zeros((count, 3), np.float32)])
    mat = np.zeros(v.shape[0], np.int32)
    par = np.full(v.shape[0], 0.2, np.float32)
    return _finish(v, alb, em, mat, par)


def batch_jobs(count: int = 64, seed: int = 0x5EED0003):
    """The batched workload's job list: per job the room plus a seeded triangle soup
    whose size is log-uniform in [1e3, 5e5] triangles, a resolution drawn from
    {256x256, 512x384, 1024x768}, log-uniform spp in [4, 64] and depth 6. Returns
    dicts with the soup's seed and size (build the scene with ``soup_scene``)."""
    idx = np.arange(count, dtype=np.uint64)
    u_n, u_r, u_s = (uniform(seed, k, idx) for k in range(3))
    sizes = ((256, 256), (512, 384), (1024, 768))
    jobs = []
    for i in range(count):
        n = int(round(math.exp(math.log(1e3) + float(u_n[i]) * math.log(5e5 / 1e3))))
        w, h = sizes[min(2, int(float(u_r[i]) * 3))]
        spp = int(round(math.exp(math.log(4.0) + float(u_s[i]) * math.log(64.0 / 4.0))))
        jobs.append({"soup_seed": seed + 1 + i, "triangles": n, "width": w, "height": h, "spp": spp,
                     "max_depth": 6})
    return jobs


def views(count: int = 16, size: int = 384, seed: int = 0x5EED0005):
    """Seeded camera views of the room for multi-view inverse rendering: each camera
    stands just inside the open front (x, y in [-1.5, 1.5] m, z in [2.0, 2.6] m) and
    looks at a point near the back wall (x, y in [-1, 1] m, z in [-2, -1] m) with a
    50 degree vertical field of view."""
    idx = np.arange(count, dtype=np.uint64)
    u = [uniform(seed, k, idx) for k in range(6)]
    out = []
    for i in range(count):
        pos = (-1.5 + 3.0 * float(u[0][i]), -1.5 + 3.0 * float(u[1][i]), 2.0 + 0.6 * float(u[2][i]))
        tgt = (-1.0 + 2.0 * float(u[3][i]), -1.0 + 2.0 * float(u[4][i]), -2.0 + float(u[5][i]))
        out.append({"position": pos, "target": tgt, "up": (0.0, 1.0, 0.0), "vfov_deg": 50.0, "width": size,
                    "height": size})
    return out


def glm_normalize(v: np.ndarray) -> np.ndarray:
    """glm::normalize in float32: v * (1 / sqrt((x*x + y*y) + z*z))."""
    v = np.asarray(v, np.float32)
    d = (v[..., 0] * v[..., 0] + v[..., 1] * v[..., 1]) + v[..., 2] * v[..., 2]
    s = np.float32(1.0) / np.sqrt(d.astype(np.float32))
    return (v * s[..., None]).astype(np.float32)
