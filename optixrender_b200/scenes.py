"""Seeded procedural scenes of the benchmark configurations.

Each generator returns a ``SceneSpec``: meshes, lights, media, an optional
equirectangular environment, a camera and render settings.  ``build_scene``
turns a spec into a ``Scene`` of the CUDA library; the CPU oracle builds its
own scene from the same arrays.  All randomness comes from
``numpy.random.default_rng(seed)``.

* ``cornell``  - 256x256, 16 spp, depth 8: five wall quads and two boxes
  (34 triangles), Lambert walls, a GGX conductor box, a ceiling quad light.
* ``spheres``  - 1920x1080, 64 spp, depth 16: a level-8 icosphere
  (1,310,720 triangles) displaced by fBm, 64 spheres of 20,000 triangles each
  (conductor / dielectric / plastic), and a 2048x1024 sky with a 0.5-degree
  sun of peak radiance 5e3.
* ``media``    - 1280x720, 256 spp, depth 32: a 128^3 fBm density grid inside
  an IOR-1.33 dielectric sphere, a homogeneous fog slab, an area light and the
  same sky.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import (FILTER_BOX, FILTER_GAUSSIAN, LIGHT_QUAD, MAT_CONDUCTOR, MAT_DIELECTRIC, MAT_DIFFUSE, MAT_METAL_WORKFLOW, MAT_PLASTIC,
               MEDIUM_GRID, MEDIUM_HOMOGENEOUS, PHASE_HG, PHASE_ISOTROPIC, RNG_PCG32, Renderer, Scene, camera,
               light, material, medium, options)


@dataclass
class MeshSpec:
    positions: np.ndarray            # (n, 3) float32
    indices: Optional[np.ndarray]    # (m, 3) int32 or None (de-indexed)
    material: dict
    out_medium: int = -1
    in_medium: int = -1
    normals: Optional[np.ndarray] = None     # (n, 3) per vertex, or None (face normals)
    texcoords: Optional[np.ndarray] = None   # (n, 2) per vertex, or None

    def _deindex(self, a, k):
        if self.indices is None:
            return np.ascontiguousarray(a.reshape(-1, 3 * k), dtype=np.float32)
        return np.ascontiguousarray(a[self.indices].reshape(-1, 3 * k), dtype=np.float32)

    def triangles(self) -> np.ndarray:
        """(m, 9) float32 de-indexed vertex positions."""
        return self._deindex(self.positions, 3)

    def tri_normals(self):
        return None if self.normals is None else self._deindex(self.normals, 3)

    def tri_texcoords(self):
        return None if self.texcoords is None else self._deindex(self.texcoords, 2)


@dataclass
class SceneSpec:
    name: str
    meshes: list
    lights: list = field(default_factory=list)      # dicts for light()
    media: list = field(default_factory=list)       # dicts for medium()
    env: Optional[np.ndarray] = None                # (h, w, 4) float32
    camera: dict = field(default_factory=dict)
    settings: dict = field(default_factory=dict)    # options() keywords
    textures: list = field(default_factory=list)    # (h, w, 4) uint8, row 0 at v = 0

    @property
    def num_triangles(self):
        return int(sum(m.triangles().shape[0] if m.indices is None else m.indices.shape[0] for m in self.meshes))


# ------------------------------------------------------------------ geometry
def box(lo, hi):
    """Axis-aligned box: 8 vertices, 12 outward-wound triangles."""
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    v = np.array([[x0, y0, z0], [x1, y0, z0], [x1, y1, z0], [x0, y1, z0],
                  [x0, y0, z1], [x1, y0, z1], [x1, y1, z1], [x0, y1, z1]], np.float32)
    f = np.array([[0, 2, 1], [0, 3, 2], [4, 5, 6], [4, 6, 7], [0, 1, 5], [0, 5, 4],
                  [3, 6, 2], [3, 7, 6], [0, 4, 7], [0, 7, 3], [1, 2, 6], [1, 6, 5]], np.int32)
    return v, f


def quad(p, u, v):
    p, u, v = (np.asarray(a, np.float32) for a in (p, u, v))
    verts = np.stack([p, p + u, p + u + v, p + v])
    return verts, np.array([[0, 1, 2], [0, 2, 3]], np.int32)


def icosphere(level):
    """Unit icosphere of 20 * 4^level triangles (shared vertices)."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], np.float64)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
                  [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], np.int64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    for _ in range(level):
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        e.sort(axis=1)
        key = e[:, 0] * (len(v) + 1) + e[:, 1]
        uniq, inv = np.unique(key, return_inverse=True)
        a = uniq // (len(v) + 1)
        b = uniq % (len(v) + 1)
        mid = v[a] + v[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = len(v)
        v = np.concatenate([v, mid])
        nf = len(f)
        m01 = base + inv[:nf]
        m12 = base + inv[nf:2 * nf]
        m20 = base + inv[2 * nf:]
        f = np.concatenate([np.stack([f[:, 0], m01, m20], 1), np.stack([f[:, 1], m12, m01], 1),
                            np.stack([f[:, 2], m20, m12], 1), np.stack([m01, m12, m20], 1)])
    return v, f


def uv_sphere(n_lat=101, n_lon=100):
    """UV sphere with 2 * n_lon * (n_lat - 1) triangles (20,000 by default)."""
    th = np.linspace(0.0, np.pi, n_lat)
    ph = np.linspace(0.0, 2 * np.pi, n_lon, endpoint=False)
    st, ct = np.sin(th)[:, None], np.cos(th)[:, None]
    v = np.stack([st * np.cos(ph)[None], ct * np.ones_like(ph)[None], st * np.sin(ph)[None]], -1).reshape(-1, 3)
    idx = np.arange(n_lat * n_lon).reshape(n_lat, n_lon)
    a = idx[:-1]
    b = np.roll(idx[:-1], -1, axis=1)
    c = idx[1:]
    d = np.roll(idx[1:], -1, axis=1)
    f = np.concatenate([np.stack([a, c, b], -1).reshape(-1, 3), np.stack([b, c, d], -1).reshape(-1, 3)])
    return v, f


def _hash3(ix, iy, iz, seed):
    with np.errstate(over="ignore"):
        return _hash3_impl(ix, iy, iz, seed)


def _hash3_impl(ix, iy, iz, seed):
    h = (ix.astype(np.uint64) * np.uint64(0x8da6b343) ^ iy.astype(np.uint64) * np.uint64(0xd8163841) ^
         iz.astype(np.uint64) * np.uint64(0xcb1ab31f) ^ np.uint64(seed) * np.uint64(0x9E3779B97F4A7C15))
    h ^= h >> np.uint64(33)
    h *= np.uint64(0xff51afd7ed558ccd)
    h ^= h >> np.uint64(33)
    h *= np.uint64(0xc4ceb9fe1a85ec53)
    h ^= h >> np.uint64(33)
    return (h >> np.uint64(40)).astype(np.float64) / float(1 << 24)


def value_noise(p, seed):
    """Trilinear value noise in [-1, 1] with smoothstep weights."""
    p = np.asarray(p, np.float64)
    i = np.floor(p).astype(np.int64)
    f = p - i
    w = f * f * (3 - 2 * f)
    out = np.zeros(p.shape[:-1])
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                h = _hash3(i[..., 0] + dx, i[..., 1] + dy, i[..., 2] + dz, seed)
                wx = w[..., 0] if dx else 1 - w[..., 0]
                wy = w[..., 1] if dy else 1 - w[..., 1]
                wz = w[..., 2] if dz else 1 - w[..., 2]
                out += wx * wy * wz * (2 * h - 1)
    return out


def fbm(p, seed, octaves=5, freq=2.0, lacunarity=2.0, gain=0.5):
    amp, total, norm = 1.0, 0.0, 0.0
    p = np.asarray(p, np.float64) * freq
    for o in range(octaves):
        total = total + amp * value_noise(p, seed + 7919 * o)
        norm += amp
        amp *= gain
        p = p * lacunarity
    return total / norm


def sky(width=2048, height=1024, sun_elev_deg=35.0, sun_azim_deg=40.0, sun_peak=5e3, sun_diam_deg=0.5):
    """Equirectangular RGBA sky: a gradient and a sun lobe.  Row r holds
    v = (r + 0.5) / height and column c holds u = (c + 0.5) / width in the
    reference's mapping (core/cuda/Sampling.h:12-33)."""
    u = (np.arange(width) + 0.5) / width
    v = (np.arange(height) + 0.5) / height
    phi = 2 * np.pi * (u - 0.5)
    th = np.pi * (v - 0.5)
    d = np.stack([np.cos(th)[:, None] * np.cos(phi)[None], np.sin(th)[:, None] * np.ones_like(phi)[None],
                  np.cos(th)[:, None] * np.sin(phi)[None]], -1)
    y = d[..., 1]
    t = np.clip(y, 0, 1)[..., None]
    horizon = np.array([0.85, 0.9, 1.0])
    zenith = np.array([0.15, 0.3, 0.75])
    ground = np.array([0.25, 0.22, 0.2])
    col = np.where((y >= 0)[..., None], horizon * (1 - t) + zenith * t, ground * (0.5 + 0.5 * (1 + y[..., None])))
    se, sa = np.radians(sun_elev_deg), np.radians(sun_azim_deg)
    s = np.array([np.cos(se) * np.cos(sa), np.sin(se), np.cos(se) * np.sin(sa)])
    ang = np.degrees(np.arccos(np.clip(d @ s, -1, 1)))
    r = sun_diam_deg / 2
    lobe = np.clip(1 - (ang / r) ** 2, 0, 1)
    col = col + sun_peak * lobe[..., None] * np.array([1.0, 0.95, 0.85])
    img = np.concatenate([col, np.ones(col.shape[:2] + (1,))], -1).astype(np.float32)
    return img


# ------------------------------------------------------------------ scenes
def cornell(width=256, height=256, spp=16, seed=1):
    white = dict(type=MAT_DIFFUSE, albedo=(0.73, 0.73, 0.73), roughness=0.0)
    red = dict(type=MAT_DIFFUSE, albedo=(0.65, 0.05, 0.05), roughness=0.0)
    green = dict(type=MAT_DIFFUSE, albedo=(0.12, 0.45, 0.15), roughness=0.0)
    copper = dict(type=MAT_CONDUCTOR, albedo=(1.0, 1.0, 1.0), roughness=0.2)
    meshes = []
    for p, u, v, m in [((0, 0, 0), (1, 0, 0), (0, 0, 1), white),     # floor
                       ((0, 1, 0), (0, 0, 1), (1, 0, 0), white),     # ceiling
                       ((0, 0, 1), (1, 0, 0), (0, 1, 0), white),     # back
                       ((0, 0, 0), (0, 0, 1), (0, 1, 0), red),       # left
                       ((1, 0, 0), (0, 1, 0), (0, 0, 1), green)]:    # right
        verts, f = quad(p, u, v)
        meshes.append(MeshSpec(verts, f, m))
    v, f = box((0.13, 0.0, 0.2), (0.43, 0.3, 0.5))
    meshes.append(MeshSpec(v, f, white))
    v, f = box((0.55, 0.0, 0.45), (0.85, 0.6, 0.75))
    meshes.append(MeshSpec(v, f, copper))
    # Quad light just below the ceiling, emitting downwards (-cross(u, v)).
    lights = [dict(type=LIGHT_QUAD, position=(0.375, 0.999, 0.375), u=(0.0, 0.0, 0.25), v=(0.25, 0.0, 0.0),
                   radiance=(17.0, 12.0, 4.0), double_side=0)]
    cam = dict(from_=(0.5, 0.5, -1.6), at=(0.5, 0.5, 0.5), up=(0, 1, 0))
    settings = dict(width=width, height=height, spp=spp, max_depth=8, rr_depth=3, rng=RNG_PCG32, seed=seed,
                    filter=FILTER_GAUSSIAN)
    return SceneSpec("cornell", meshes, lights, [], None, cam, settings)


def portal(width=96, height=96, spp=16, seed=1):
    """A closed diffuse room split by a wall with a 0.2 x 0.2 opening; the only
    light (a quad under the ceiling, facing down) is behind the wall, so the
    camera's half of the room (dark grey surfaces) is lit through the opening
    by the bright walls of the far half: next-event estimation rarely connects
    and cosine-weighted BSDF sampling rarely finds the opening, the case a
    learned proposal is for."""
    bright = dict(type=MAT_DIFFUSE, albedo=(0.8, 0.8, 0.8), roughness=0.0)
    warm = dict(type=MAT_DIFFUSE, albedo=(0.85, 0.65, 0.45), roughness=0.0)
    dark = dict(type=MAT_DIFFUSE, albedo=(0.3, 0.3, 0.3), roughness=0.0)
    meshes = []
    # the camera's half (z < 0.5) is dark grey, the lit half bright
    for z0, z1, m in [(0.0, 0.5, dark), (0.5, 1.0, bright)]:
        dz = z1 - z0
        for p, u, v in [((0, 0, z0), (1, 0, 0), (0, 0, dz)),      # floor (normal +y)
                        ((0, 1, z0), (0, 0, dz), (1, 0, 0)),      # ceiling (-y)
                        ((0, 0, z0), (0, 0, dz), (0, 1, 0)),      # left (+x)
                        ((1, 0, z0), (0, 1, 0), (0, 0, dz))]:     # right (-x)
            verts, f = quad(p, u, v)
            meshes.append(MeshSpec(verts, f, m))
    for p, u, v, m in [((0, 0, 1), (1, 0, 0), (0, 1, 0), warm),   # back wall, facing the room
                       ((0, 0, 0), (0, 1, 0), (1, 0, 0), dark)]:  # front wall
        verts, f = quad(p, u, v)
        meshes.append(MeshSpec(verts, f, m))
    # divider at z = 0.5 with an opening x in [0.4, 0.6], y in [0.4, 0.6]
    z = 0.5
    for (x0, x1, y0, y1) in [(0.0, 1.0, 0.0, 0.4), (0.0, 1.0, 0.6, 1.0), (0.0, 0.4, 0.4, 0.6), (0.6, 1.0, 0.4, 0.6)]:
        verts, f = quad((x0, y0, z), (x1 - x0, 0, 0), (0, y1 - y0, 0))   # facing +z (the lit half)
        meshes.append(MeshSpec(verts, f, bright))
        verts, f = quad((x0, y0, z), (0, y1 - y0, 0), (x1 - x0, 0, 0))   # facing -z (the camera)
        meshes.append(MeshSpec(verts, f, dark))
    lights = [dict(type=LIGHT_QUAD, position=(0.35, 0.999, 0.7), u=(0.0, 0.0, 0.2), v=(0.3, 0.0, 0.0),
                   radiance=(40.0, 36.0, 30.0), double_side=0)]
    # looking down at the floor and walls of the dark half, which see the opening
    cam = dict(from_=(0.5, 0.9, 0.03), at=(0.5, 0.0, 0.4), up=(0, 1, 0), fov_y_deg=0.0)
    settings = dict(width=width, height=height, spp=spp, max_depth=8, rr_depth=3, rng=RNG_PCG32, seed=seed,
                    filter=FILTER_BOX)
    return SceneSpec("portal", meshes, lights, [], None, cam, settings)


def textured(width=128, height=128, spp=16, seed=1):
    """The Cornell room with material textures: a checker albedo on the floor
    (uv repeated 3x, wrap), a bump normal map on the back wall, a roughness
    ramp on the conductor box and albedo + metallic maps on a metal-workflow
    panel.  Every mesh carries per-vertex normals and texcoords."""
    rng = np.random.default_rng(seed + 17)
    n = 64
    yy, xx = np.mgrid[0:n, 0:n]
    checker = np.where(((xx // 8) + (yy // 8)) % 2 == 0, 0, 1)[..., None]
    albedo_tex = np.where(checker == 0, np.uint8([200, 190, 170, 255]), np.uint8([40, 70, 140, 255])).astype(np.uint8)
    ramp = np.zeros((32, 32, 4), np.uint8)
    ramp[..., 0] = np.linspace(60, 230, 32, dtype=np.float64)[None, :].round().astype(np.uint8)
    ramp[..., 3] = 255
    # normal map: height field h = 0.15 sin(2pi x/16) sin(2pi y/16), n = normalize(-dh/dx, -dh/dy, 1)
    ph = 2 * np.pi / 16.0
    dhdx = 0.15 * ph * np.cos(ph * xx) * np.sin(ph * yy) * 8
    dhdy = 0.15 * ph * np.sin(ph * xx) * np.cos(ph * yy) * 8
    nrm = np.stack([-dhdx, -dhdy, np.ones_like(dhdx)], -1)
    nrm /= np.linalg.norm(nrm, axis=-1, keepdims=True)
    normal_tex = np.concatenate([np.clip((nrm * 0.5 + 0.5) * 255 + 0.5, 0, 255).astype(np.uint8),
                                 np.full((n, n, 1), 255, np.uint8)], -1)
    metal_tex = np.zeros((16, 16, 4), np.uint8)
    metal_tex[..., 0] = rng.integers(0, 256, (16, 16))
    metal_tex[..., 3] = 255
    textures = [albedo_tex, ramp, normal_tex, metal_tex]

    def tquad(p, u, v, mat, uv_scale=1.0):
        verts, f = quad(p, u, v)
        nr = np.cross(np.asarray(u, np.float64), np.asarray(v, np.float64))
        nr = np.tile((nr / np.linalg.norm(nr)).astype(np.float32), (4, 1))
        uv = np.float32([[0, 0], [1, 0], [1, 1], [0, 1]]) * uv_scale
        return MeshSpec(verts, f, mat, normals=nr, texcoords=uv)

    white = dict(type=MAT_DIFFUSE, albedo=(0.73, 0.73, 0.73), roughness=0.0)
    floor = dict(type=MAT_DIFFUSE, albedo=(0.5, 0.5, 0.5), roughness=0.0, texture_ids=[0])
    back = dict(type=MAT_DIFFUSE, albedo=(0.73, 0.73, 0.73), roughness=0.0, texture_ids=[-1] * 7 + [2])
    red = dict(type=MAT_DIFFUSE, albedo=(0.65, 0.05, 0.05), roughness=0.0)
    green = dict(type=MAT_DIFFUSE, albedo=(0.12, 0.45, 0.15), roughness=0.0)
    copper = dict(type=MAT_CONDUCTOR, albedo=(1.0, 1.0, 1.0), roughness=0.2, texture_ids=[-1, 1])
    panel = dict(type=MAT_METAL_WORKFLOW, albedo=(0.8, 0.8, 0.8), roughness=0.3, texture_ids=[0, -1, -1, -1, 3])
    meshes = [tquad((0, 0, 0), (1, 0, 0), (0, 0, 1), floor, 3.0),
              tquad((0, 1, 0), (0, 0, 1), (1, 0, 0), white),
              tquad((0, 0, 1), (1, 0, 0), (0, 1, 0), back, 2.0),
              tquad((0, 0, 0), (0, 0, 1), (0, 1, 0), red),
              tquad((1, 0, 0), (0, 1, 0), (0, 0, 1), green),
              tquad((0.1, 0.05, 0.35), (0.35, 0.0, -0.1), (0.0, 0.45, 0.1), panel)]
    v, f = box((0.55, 0.0, 0.45), (0.85, 0.6, 0.75))
    # de-indexed box with face normals and planar texcoords (x + y, z)
    tv = v[f.reshape(-1)]
    e1, e2 = tv[1::3] - tv[0::3], tv[2::3] - tv[0::3]
    fn = np.cross(e1, e2)
    fn /= np.linalg.norm(fn, axis=1, keepdims=True)
    bn = np.repeat(fn, 3, axis=0).astype(np.float32)
    buv = np.stack([(tv[:, 0] - 0.55) / 0.3 + tv[:, 1], (tv[:, 2] - 0.45) / 0.3], -1).astype(np.float32)
    meshes.append(MeshSpec(tv.astype(np.float32), None, copper, normals=bn, texcoords=buv))
    lights = [dict(type=LIGHT_QUAD, position=(0.375, 0.999, 0.375), u=(0.0, 0.0, 0.25), v=(0.25, 0.0, 0.0),
                   radiance=(17.0, 12.0, 4.0), double_side=0)]
    cam = dict(from_=(0.5, 0.5, -1.6), at=(0.5, 0.5, 0.5), up=(0, 1, 0))
    settings = dict(width=width, height=height, spp=spp, max_depth=8, rr_depth=3, rng=RNG_PCG32, seed=seed,
                    filter=FILTER_GAUSSIAN)
    return SceneSpec("textured", meshes, lights, [], None, cam, settings, textures)


def spheres(width=1920, height=1080, spp=64, seed=1, ico_level=8, sphere_tris=True, env_size=(2048, 1024)):
    rng = np.random.default_rng(seed)
    v, f = icosphere(ico_level)
    disp = fbm(v * 1.5, seed, octaves=6)
    v = v * (1.0 + 0.05 * disp)[:, None]
    base = dict(type=MAT_PLASTIC, albedo=(0.55, 0.55, 0.6), roughness=0.3, int_ior=1.5, ext_ior=1.0)
    meshes = [MeshSpec(v.astype(np.float32), f.astype(np.int32), base)]
    sv, sf = uv_sphere() if sphere_tris else uv_sphere(9, 10)
    centers = []
    while len(centers) < 64:
        r = rng.uniform(0.12, 0.28)
        ang = rng.uniform(0, 2 * np.pi)
        dist = rng.uniform(1.35, 2.6)
        y = rng.uniform(-1.1, 1.1)
        c = np.array([dist * np.cos(ang), y, dist * np.sin(ang)])
        if all(np.linalg.norm(c - c2) > r + r2 + 0.02 for c2, r2 in centers):
            centers.append((c, r))
    for c, r in centers:
        kind = rng.integers(0, 3)
        if kind == 0:
            m = dict(type=MAT_CONDUCTOR, albedo=(1, 1, 1), roughness=float(rng.uniform(0.05, 0.8)),
                     eta=tuple(rng.uniform(0.2, 1.5, 3)), k=tuple(rng.uniform(2.0, 4.0, 3)))
        elif kind == 1:
            # roughness 0 makes the reference's GGX density 0/0; 0.02 is the defined minimum
            m = dict(type=MAT_DIELECTRIC, albedo=(1, 1, 1), roughness=float(max(rng.uniform(0.0, 0.3), 0.02)),
                     int_ior=1.5, ext_ior=1.0)
        else:
            m = dict(type=MAT_PLASTIC, albedo=tuple(rng.uniform(0.1, 0.9, 3)), int_ior=1.5, ext_ior=1.0)
        meshes.append(MeshSpec((sv * r + c).astype(np.float32), sf.astype(np.int32), m))
    env = sky(*env_size)
    cam = dict(from_=(0.0, 0.9, -5.2), at=(0.0, 0.0, 0.0), up=(0, 1, 0))
    settings = dict(width=width, height=height, spp=spp, max_depth=16, rr_depth=0, rng=RNG_PCG32, seed=seed,
                    filter=FILTER_GAUSSIAN)
    return SceneSpec("spheres", meshes, [], [], env, cam, settings)


def density_grid(res=128, seed=1, sigma_max=5.0):
    """A res^3 fBm density in [0, sigma_max] shaped to a ball (x fastest)."""
    ax = (np.arange(res) + 0.5) / res * 2.0 - 1.0
    z, y, x = np.meshgrid(ax, ax, ax, indexing="ij")
    p = np.stack([x, y, z], -1)
    n = fbm(p * 1.3, seed + 17, octaves=5)
    r = np.sqrt(x * x + y * y + z * z)
    ball = np.clip((1.0 - r) / 0.15, 0.0, 1.0)
    d = np.clip(0.5 + 1.2 * n, 0.0, 1.0) * ball
    return (d * sigma_max).astype(np.float32)


def media(width=1280, height=720, spp=256, seed=1, grid_res=128, env_size=(2048, 1024)):
    """A 128^3 fBm grid medium (sigma_t 0-5, albedo 0.9, HG g=0.6) inside an
    IOR-1.33 dielectric sphere; a homogeneous fog box (sigma_t 0.05, albedo
    0.9) bounded by an index-matched thin dielectric; a diffuse floor and a
    quad light inside the fog; the sky outside."""
    FOG, GRID = 0, 1
    meshes = []
    sv, sf = uv_sphere(61, 60)
    meshes.append(MeshSpec(sv.astype(np.float32), sf.astype(np.int32),
                           dict(type=MAT_DIELECTRIC, albedo=(1, 1, 1), roughness=0.05, int_ior=1.33, ext_ior=1.0),
                           out_medium=FOG, in_medium=GRID))
    lo, hi = (-3.0, -1.2, -3.0), (3.0, 2.6, 3.0)
    v, f = box(lo, hi)
    boundary = dict(type=5, albedo=(1, 1, 1), roughness=0.01, int_ior=1.0, ext_ior=1.0)  # thin dielectric, IOR 1
    keep = np.array([i for i in range(12) if i not in (4, 5)])  # faces 4,5 are the y = lo floor
    meshes.append(MeshSpec(v, f[keep], boundary, out_medium=-1, in_medium=FOG))
    fv, ff = quad((lo[0], lo[1], lo[2]), (hi[0] - lo[0], 0, 0), (0, 0, hi[2] - lo[2]))
    meshes.append(MeshSpec(fv, ff, dict(type=MAT_DIFFUSE, albedo=(0.6, 0.6, 0.6), roughness=0.0),
                           out_medium=FOG, in_medium=FOG))
    lights = [dict(type=LIGHT_QUAD, position=(-0.75, 2.4, -0.75), u=(0.0, 0.0, 1.5), v=(1.5, 0.0, 0.0),
                   radiance=(12.0, 11.0, 9.0), double_side=0, medium=FOG)]
    dens = density_grid(grid_res, seed)
    med = [dict(type=MEDIUM_HOMOGENEOUS, phase=PHASE_ISOTROPIC, sigma_s=(0.045, 0.045, 0.045),
                sigma_a=(0.005, 0.005, 0.005), scale=1.0),
           dict(type=MEDIUM_GRID, density=dens, phase=PHASE_HG, g=(0.6, 0.6, 0.6), sigma_s=(0.9, 0.9, 0.9),
                sigma_a=(0.1, 0.1, 0.1), scale=1.0, bounds_min=(-1, -1, -1), bounds_max=(1, 1, 1),
                majorant_res=8)]
    env = sky(*env_size)
    cam = dict(from_=(0.0, 0.6, -7.5), at=(0.0, 0.2, 0.0), up=(0, 1, 0), medium=-1)
    settings = dict(width=width, height=height, spp=spp, max_depth=32, rr_depth=0, rng=RNG_PCG32, seed=seed,
                    filter=FILTER_GAUSSIAN)
    return SceneSpec("media", meshes, lights, med, env, cam, settings)


def _material_obj(d):
    return material(**d)


def build_scene(spec: SceneSpec) -> Scene:
    """A CUDA-library Scene holding the spec's meshes, lights, media and sky."""
    s = Scene()
    for t in spec.textures:
        s.add_texture(t)
    for m in spec.meshes:
        s.add_mesh(m.positions, _material_obj(m.material), indices=m.indices, normals=m.normals,
                   texcoords=m.texcoords, out_medium=m.out_medium, in_medium=m.in_medium)
    for l in spec.lights:
        s.add_light(light(**l))
    for md in spec.media:
        s.add_medium(medium(**md))
    if spec.env is not None:
        s.add_env(spec.env)
    return s


def build_renderer(spec: SceneSpec, **overrides) -> tuple:
    s = build_scene(spec)
    st = dict(spec.settings)
    st.update(overrides)
    r = Renderer(s, options(**st))
    r.set_camera(camera(**spec.camera))
    return s, r


SCENES = {"cornell": cornell, "spheres": spheres, "media": media, "textured": textured, "portal": portal}
