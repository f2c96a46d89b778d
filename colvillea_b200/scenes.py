"""Seeded synthetic scenes for the benchmark configurations.

The reference's sample assets (sphere.obj, venice_sunset_2k.hdr,
src/colvillea/colvillea.cpp:62,68) are not in its repository, so the
workloads are generated here, deterministically from a seed:

  cfg1  256x256, 16 spp, depth 5, RR from 3: 20x20 ground quad (2 tris) +
        32 icospheres (subdivision 2, 320 tris), 256x128 HDRI + directional.
  cfg2  1920x1080, 64 spp, depth 8, RR from 3: 1024x1024-vertex fBm terrain
        (2,093,058 tris) + 512 icosphere/torus meshes (~5k tris each),
        2048x1024 HDRI (8 lobes, peak 200) + directional.
  cfg3  cfg1 scene at 1920x1080, 128 spp.
  cfg4  cfg1 geometry with 60% rough dielectric (alpha U[0.01,0.1]),
        2048x1024 HDRI with one lobe (peak 5000, sigma 0.5 deg).
  cfg5  3840x2160, 256 spp, depth 16: 2048x2048-vertex terrain + 128 unique
        meshes x 12 instances with random rotations and scales U[0.5, 2].

Every mesh carries per-vertex normals, tangents and uvs (the reference
requires tangents, src/core/devices/optix.cu:187-188).  A `Scene` holds the
meshes, instances (entities), materials, emitters and camera in the
reference's units and can be flattened to world-space arrays (`flatten`).
"""
import functools
import math
from dataclasses import dataclass, field

import numpy as np

MAT_DIFFUSE, MAT_METAL, MAT_GLASS = 0, 1, 2
EMIT_DIRECTIONAL, EMIT_DOME = 0, 1
GOLD_ETA = (0.143119, 0.374957, 1.442479)
GOLD_K = (3.983160, 2.385721, 1.603215)
IDENTITY = (1.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0)


@dataclass
class Mesh:
    positions: np.ndarray  # (nv, 3) float32
    normals: np.ndarray    # (nv, 3) float32 or None
    tangents: np.ndarray   # (nv, 3) float32
    uvs: np.ndarray        # (nv, 2) float32 or None
    indices: np.ndarray    # (nt, 3) uint32


@dataclass
class Material:
    type: int
    reflectance: tuple = (0.0, 0.0, 0.0)
    roughness: float = 0.0
    interior_ior: float = 1.5
    eta: tuple = (0.0, 0.0, 0.0)
    k: tuple = (0.0, 0.0, 0.0)
    reflectance_texture: int = 0   # 1-based index into Scene.textures, 0 = none
    roughness_texture: int = 0
    normal_texture: int = 0

    def as_array(self):
        return np.array([self.type, *self.reflectance, self.roughness, self.interior_ior, *self.eta, *self.k,
                         self.reflectance_texture, self.roughness_texture, self.normal_texture, 0], np.float32)


TEX_RGBA8, TEX_RGBA32F = 0, 1


@dataclass
class Texture:
    """An image texture: (h, w, 4) uint8 (RGBA8, optionally sRGB) or float32 (RGBA32F)."""
    texels: np.ndarray
    srgb: bool = False

    @property
    def format(self):
        return TEX_RGBA8 if self.texels.dtype == np.uint8 else TEX_RGBA32F


@dataclass
class Emitter:
    type: int
    intensity: tuple = (0.0, 0.0, 0.0)
    direction: tuple = (0.0, -1.0, 0.0)
    angular_radius: float = 0.0
    texels: np.ndarray = None  # (h, w, 4) float32

    def as_array(self):
        w = h = 0
        if self.texels is not None:
            h, w = self.texels.shape[:2]
        return np.array([self.type, *self.intensity, *self.direction, self.angular_radius, w, h, 0, 0], np.float32)


@dataclass
class Scene:
    width: int
    height: int
    meshes: list
    instances: list          # (mesh_id, material_index, transform 12 floats)
    materials: list
    emitters: list
    camera: np.ndarray       # (12,) pos, d00, ddu, ddv
    spp: int = 16
    max_depth: int = 5
    rr_start: int = 3
    name: str = ""
    info: dict = field(default_factory=dict)
    textures: list = field(default_factory=list)

    @property
    def num_triangles(self):
        return sum(len(self.meshes[m].indices) for m, _, _ in self.instances)

    def dome(self):
        for e in reversed(self.emitters):
            if e.type == EMIT_DOME:
                return e
        return None

    def flatten(self):
        """World-space arrays in instance order (the order of global triangle ids)."""
        pos, nrm, tan, uv, idx, tm = [], [], [], [], [], []
        base = 0
        for mesh_id, mat, xf in self.instances:
            m = self.meshes[mesh_id]
            # the integrator receives the transform as float32 (cl_instance_desc)
            M = np.asarray(xf, np.float32).astype(np.float64).reshape(3, 4)
            if np.array_equal(M, np.asarray(IDENTITY).reshape(3, 4)):
                p, n, t = m.positions, m.normals, m.tangents
            else:
                L = M[:, :3]
                p = (m.positions.astype(np.float64) @ L.T + M[:, 3]).astype(np.float32)
                t = (m.tangents.astype(np.float64) @ L.T).astype(np.float32)
                n = (m.normals.astype(np.float64) @ np.linalg.inv(L)).astype(np.float32)
            pos.append(p); nrm.append(n); tan.append(t); uv.append(m.uvs)
            idx.append(m.indices.astype(np.uint32) + np.uint32(base))
            tm.append(np.full(len(m.indices), mat, np.uint32))
            base += len(m.positions)
        dome = self.dome()
        return FlatScene(
            pos=np.concatenate(pos), nrm=np.concatenate(nrm), tan=np.concatenate(tan), uv=np.concatenate(uv),
            idx=np.concatenate(idx), tri_material=np.concatenate(tm),
            materials=np.stack([m.as_array() for m in self.materials]),
            emitters=np.stack([e.as_array() for e in self.emitters]) if self.emitters else np.zeros((0, 12), np.float32),
            dome_texels=dome.texels if dome is not None else np.zeros((1, 1, 4), np.float32),
            camera=np.asarray(self.camera, np.float32), width=self.width, height=self.height,
            textures=list(self.textures))


@dataclass
class FlatScene:
    pos: np.ndarray
    nrm: np.ndarray
    tan: np.ndarray
    uv: np.ndarray
    idx: np.ndarray
    tri_material: np.ndarray
    materials: np.ndarray
    emitters: np.ndarray
    dome_texels: np.ndarray
    camera: np.ndarray
    width: int
    height: int
    textures: list = field(default_factory=list)


# ---------------------------------------------------------------------------
# Geometry
# ---------------------------------------------------------------------------
def _frame_from_normal(n):
    """Unit tangent perpendicular to n, along the longitude direction."""
    up = np.zeros_like(n); up[:, 1] = 1.0
    t = np.cross(up, n)
    bad = np.linalg.norm(t, axis=1) < 1e-6
    t[bad] = np.array([1.0, 0.0, 0.0])
    return t / np.linalg.norm(t, axis=1, keepdims=True)


@functools.lru_cache(maxsize=8)
def icosphere(subdiv):
    """Unit icosphere: (positions, indices) float64/uint32 (cached; do not modify)."""
    p = (1.0 + 5 ** 0.5) / 2.0
    v = [(-1, p, 0), (1, p, 0), (-1, -p, 0), (1, -p, 0), (0, -1, p), (0, 1, p), (0, -1, -p), (0, 1, -p),
         (p, 0, -1), (p, 0, 1), (-p, 0, -1), (-p, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
         (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
         (8, 6, 7), (9, 8, 1)]
    verts = [np.array(x, np.float64) / np.linalg.norm(x) for x in v]
    faces = f
    for _ in range(subdiv):
        cache = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    v_out, f_out = np.array(verts), np.array(faces, np.uint32)
    v_out.flags.writeable = False
    f_out.flags.writeable = False
    return v_out, f_out


def sphere_mesh(subdiv, center, radius):
    v, f = icosphere(subdiv)
    n = v.copy()
    pos = v * radius + np.asarray(center)
    t = _frame_from_normal(n)
    uv = np.stack([np.arctan2(n[:, 0], n[:, 2]) / (2 * np.pi) + 0.5, np.arccos(np.clip(n[:, 1], -1, 1)) / np.pi], 1)
    return Mesh(pos.astype(np.float32), n.astype(np.float32), t.astype(np.float32), uv.astype(np.float32), f)


def torus_mesh(nu, nv, center, R, r):
    u = np.arange(nu) * 2 * np.pi / nu
    w = np.arange(nv) * 2 * np.pi / nv
    U, V = np.meshgrid(u, w, indexing="ij")
    cu, su, cv, sv = np.cos(U), np.sin(U), np.cos(V), np.sin(V)
    pos = np.stack([(R + r * cv) * cu, r * sv, (R + r * cv) * su], -1).reshape(-1, 3)
    nrm = np.stack([cv * cu, sv, cv * su], -1).reshape(-1, 3)
    tan = np.stack([-su, np.zeros_like(su), cu], -1).reshape(-1, 3)
    uv = np.stack([U / (2 * np.pi), V / (2 * np.pi)], -1).reshape(-1, 2)
    i = np.arange(nu)[:, None]; j = np.arange(nv)[None, :]
    a = (i * nv + j); b = ((i + 1) % nu) * nv + j; c = ((i + 1) % nu) * nv + (j + 1) % nv; d = i * nv + (j + 1) % nv
    idx = np.concatenate([np.stack([a, b, c], -1).reshape(-1, 3), np.stack([a, c, d], -1).reshape(-1, 3)])
    return Mesh((pos + np.asarray(center)).astype(np.float32), nrm.astype(np.float32), tan.astype(np.float32),
                uv.astype(np.float32), idx.astype(np.uint32))


def quad_mesh(size, y=0.0, uv_scale=1.0):
    h = size / 2.0
    pos = np.array([[-h, y, -h], [h, y, -h], [h, y, h], [-h, y, h]], np.float32)
    nrm = np.tile(np.array([0, 1, 0], np.float32), (4, 1))
    tan = np.tile(np.array([1, 0, 0], np.float32), (4, 1))
    uv = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32) * np.float32(uv_scale)
    idx = np.array([[0, 2, 1], [0, 3, 2]], np.uint32)
    return Mesh(pos, nrm, tan, uv, idx)


def _value_noise(x, z, rng_seed):
    """2-D value noise on the integer lattice, smoothstep-interpolated."""
    xi, zi = np.floor(x).astype(np.int64), np.floor(z).astype(np.int64)
    fx, fz = x - xi, z - zi

    def h(a, b):
        k = (a * 73856093) ^ (b * 19349663) ^ (rng_seed * 83492791)
        k = (k ^ (k >> 13)) * 1274126177
        k = k ^ (k >> 16)
        return (k & 0xFFFF).astype(np.float64) / 65535.0 * 2.0 - 1.0

    sx, sz = fx * fx * (3 - 2 * fx), fz * fz * (3 - 2 * fz)
    a = h(xi, zi) * (1 - sx) + h(xi + 1, zi) * sx
    b = h(xi, zi + 1) * (1 - sx) + h(xi + 1, zi + 1) * sx
    return a * (1 - sz) + b * sz


def terrain_mesh(n, extent, amplitude, octaves, seed, y0=0.0):
    """n x n vertex fBm heightfield over [-extent, extent]^2."""
    s = np.linspace(-extent, extent, n)
    X, Z = np.meshgrid(s, s, indexing="xy")
    Hh = np.zeros_like(X)
    freq, amp, norm = 4.0 / (2 * extent), 1.0, 0.0
    for o in range(octaves):
        Hh += amp * _value_noise(X * freq + 17.3 * o, Z * freq - 9.1 * o, seed + o)
        norm += amp
        freq *= 2.0
        amp *= 0.5
    Hh = Hh / norm * amplitude + y0
    pos = np.stack([X, Hh, Z], -1).reshape(-1, 3)
    dx = np.gradient(Hh, s, axis=1)
    dz = np.gradient(Hh, s, axis=0)
    nrm = np.stack([-dx, np.ones_like(dx), -dz], -1).reshape(-1, 3)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    tan = np.stack([np.ones_like(dx), dx, np.zeros_like(dx)], -1).reshape(-1, 3)
    tan /= np.linalg.norm(tan, axis=1, keepdims=True)
    uv = np.stack([(X + extent) / (2 * extent), (Z + extent) / (2 * extent)], -1).reshape(-1, 2)
    i = np.arange(n - 1)[:, None]; j = np.arange(n - 1)[None, :]
    a = i * n + j; b = a + 1; c = a + n + 1; d = a + n
    idx = np.concatenate([np.stack([a, c, b], -1).reshape(-1, 3), np.stack([a, d, c], -1).reshape(-1, 3)])
    return Mesh(pos.astype(np.float32), nrm.astype(np.float32), tan.astype(np.float32), uv.astype(np.float32),
                idx.astype(np.uint32))


# ---------------------------------------------------------------------------
# Lights and camera
# ---------------------------------------------------------------------------
def texel_directions(w, h):
    """Direction of each texel centre (hdridome.h:207-222 mapping)."""
    u = (np.arange(w) + 0.5) / w
    v = (np.arange(h) + 0.5) / h
    U, V = np.meshgrid(u, v, indexing="xy")
    th, ph = np.pi * V, -2 * np.pi * (U - 0.5)
    return np.stack([np.sin(th) * np.sin(ph), np.cos(th), np.sin(th) * np.cos(ph)], -1)


def hdri(w, h, lobes, rng, zenith=(0.3, 0.5, 1.0), horizon=(1.0, 1.0, 1.0)):
    """Vertical sky gradient (zenith to horizon; lower hemisphere = horizon)
    plus Gaussian lobes [(direction, sigma_deg, peak)], RGBA32F (h, w, 4)."""
    d = texel_directions(w, h)
    t = np.clip(d[..., 1], 0.0, 1.0)[..., None]
    sky = np.asarray(horizon) * (1 - t) + np.asarray(zenith) * t
    for dirv, sigma_deg, peak in lobes:
        dirv = np.asarray(dirv, np.float64) / np.linalg.norm(dirv)
        ang = np.arccos(np.clip(d @ dirv, -1.0, 1.0))
        sig = math.radians(sigma_deg)
        sky = sky + peak * np.exp(-ang * ang / (2 * sig * sig))[..., None]
    out = np.ones((h, w, 4), np.float32)
    out[..., :3] = sky
    return out


def random_upper_dirs(rng, n, min_y=0.15):
    out = []
    while len(out) < n:
        v = rng.normal(size=3)
        v /= np.linalg.norm(v)
        if v[1] > min_y:
            out.append(v)
    return out


def directional(irradiance=3.0, radius_deg=0.5, direction=(-0.35, -1.0, 0.45)):
    """Sun disk: the reference's directional value is radiance over a cone of
    the angular radius (directional.h:36-54), so intensity = E / (pi tan^2 r)."""
    r = math.radians(radius_deg)
    L = irradiance / (math.pi * math.tan(r) ** 2)
    d = np.asarray(direction, np.float64)
    d /= np.linalg.norm(d)
    return Emitter(EMIT_DIRECTIONAL, (L, L, L), tuple(float(x) for x in d), r)


def look_at_camera(pos, at, up, fov_deg, width, height):
    """(pos, d00, ddu, ddv) of a pinhole camera (camera.h:8-27): pixel (x, y)
    looks along d00 + (x/W) ddu + (y/H) ddv; y grows downwards."""
    pos, at, up = (np.asarray(a, np.float64) for a in (pos, at, up))
    f = at - pos
    f /= np.linalg.norm(f)
    r = np.cross(f, up); r /= np.linalg.norm(r)
    u = np.cross(r, f)
    hh = 2.0 * math.tan(math.radians(fov_deg) / 2.0)
    ww = hh * width / height
    ddu = r * ww
    ddv = -u * hh
    d00 = f - 0.5 * ddu - 0.5 * ddv
    return np.concatenate([pos, d00, ddu, ddv]).astype(np.float32)


def _random_material(rng, glass_frac=None, glass_alpha=(0.05, 0.3)):
    if glass_frac is not None:
        kind = MAT_GLASS if rng.random() < glass_frac else int(rng.integers(0, 2))
    else:
        kind = int(rng.integers(0, 3))
    if kind == MAT_DIFFUSE:
        return Material(MAT_DIFFUSE, reflectance=tuple(float(x) for x in rng.uniform(0.2, 0.8, 3)))
    if kind == MAT_METAL:
        a = rng.uniform(0.05, 0.5)
        return Material(MAT_METAL, reflectance=(1.0, 1.0, 1.0), roughness=float(math.sqrt(a)), eta=GOLD_ETA, k=GOLD_K)
    a = rng.uniform(*glass_alpha)
    return Material(MAT_GLASS, roughness=float(math.sqrt(a)), interior_ior=1.5)


# ---------------------------------------------------------------------------
# Procedural textures (seeded)
# ---------------------------------------------------------------------------
def _smooth_noise(n, cells, rng):
    """(n, n) periodic value noise in [0, 1] (bilinear over a cells x cells lattice)."""
    g = rng.random((cells, cells))
    x = np.arange(n) * cells / n
    i0 = np.floor(x).astype(int); f = x - i0; i1 = (i0 + 1) % cells
    f = f * f * (3 - 2 * f)
    a = g[i0][:, i0] * (1 - f)[None, :] + g[i0][:, i1] * f[None, :]
    b = g[i1][:, i0] * (1 - f)[None, :] + g[i1][:, i1] * f[None, :]
    return a * (1 - f)[:, None] + b * f[:, None]


def checker_texture(n, squares, c0, c1, rng, srgb=True):
    """RGBA8 checkerboard with noise, sRGB-encoded colours."""
    y, x = np.mgrid[0:n, 0:n]
    m = ((x * squares // n + y * squares // n) % 2)[..., None]
    c = np.where(m == 1, np.asarray(c1, np.float64), np.asarray(c0, np.float64))
    c = np.clip(c * (0.75 + 0.5 * _smooth_noise(n, 8, rng))[..., None], 0, 1)
    out = np.empty((n, n, 4), np.uint8)
    out[..., :3] = np.round(c * 255)
    out[..., 3] = 255
    return Texture(out, srgb=srgb)


def color_texture(n, rng):
    """RGBA32F smooth colours in [0.05, 0.95]."""
    out = np.ones((n, n, 4), np.float32)
    for c in range(3):
        out[..., c] = 0.05 + 0.9 * _smooth_noise(n, 6, rng)
    return Texture(out)


def roughness_texture(n, rng, lo=0.05, hi=0.8):
    """RGBA8 linear: roughness in the red channel."""
    r = lo + (hi - lo) * _smooth_noise(n, 5, rng)
    out = np.zeros((n, n, 4), np.uint8)
    out[..., 0] = np.round(r * 255)
    out[..., 3] = 255
    return Texture(out)


def normal_map(n, rng, tilt=0.5, cells=12):
    """RGBA8 linear tangent-space normal map of a periodic height field:
    n = normalize(-k dh/du, -k dh/dv, 1) with k setting the slopes' standard
    deviation to `tilt`, stored as (n + 1) / 2."""
    h = _smooth_noise(n, cells, rng)
    du = np.roll(h, -1, 1) - np.roll(h, 1, 1)
    dv = np.roll(h, -1, 0) - np.roll(h, 1, 0)
    k = tilt / max(np.std(np.concatenate([du.ravel(), dv.ravel()])), 1e-12)
    v = np.stack([-k * du, -k * dv, np.ones_like(h)], -1)
    v /= np.linalg.norm(v, axis=-1, keepdims=True)
    out = np.zeros((n, n, 4), np.uint8)
    out[..., :3] = np.round((v + 1) * 0.5 * 255)
    out[..., 3] = 255
    return Texture(out)


# ---------------------------------------------------------------------------
# Configurations
# ---------------------------------------------------------------------------
def config1(seed=0, width=256, height=256, glass_frac=None, glass_alpha=(0.05, 0.3), dome=None):
    rng = np.random.default_rng(seed)
    meshes, inst, mats = [quad_mesh(20.0)], [(0, 0, IDENTITY)], [Material(MAT_DIFFUSE, reflectance=(0.5, 0.5, 0.5))]
    for i in range(32):
        r = rng.uniform(0.2, 0.6)
        c = (rng.uniform(-4, 4), rng.uniform(0.2, 2.0), rng.uniform(-4, 4))
        meshes.append(sphere_mesh(2, c, r))
        mats.append(_random_material(rng, glass_frac, glass_alpha))
        inst.append((len(meshes) - 1, len(mats) - 1, IDENTITY))
    if dome is None:
        lobes = [(d, 2.0, 50.0) for d in random_upper_dirs(rng, 3)]
        dome = Emitter(EMIT_DOME, texels=hdri(256, 128, lobes, rng))
    ems = [directional(), dome]
    cam = look_at_camera((0, 3, -10), (0, 0, 0), (0, 1, 0), 45.0, width, height)
    return Scene(width, height, meshes, inst, mats, ems, cam, spp=16, max_depth=5, rr_start=3, name="cfg1")


def textured(seed=0, width=256, height=256):
    """Config 1's layout with image textures on every material kind: an sRGB
    checker and a normal map on the ground, RGBA32F reflectance textures,
    metal reflectance and roughness textures, normal maps on metal and glass
    spheres."""
    rng = np.random.default_rng(seed + 31)
    tex = [checker_texture(256, 8, (0.8, 0.75, 0.7), (0.15, 0.2, 0.3), rng),   # 1 ground albedo (sRGB)
           normal_map(256, rng),                                                # 2 ground bumps
           color_texture(64, rng), color_texture(128, rng),                     # 3, 4 diffuse colours
           roughness_texture(64, rng),                                          # 5 metal roughness
           checker_texture(64, 4, (1.0, 0.85, 0.6), (0.9, 0.9, 0.95), rng, srgb=False),  # 6 metal reflectance
           normal_map(128, rng, tilt=0.8, cells=6)]                         # 7 sphere bumps
    meshes = [quad_mesh(20.0, uv_scale=4.0)]
    mats = [Material(MAT_DIFFUSE, reflectance=(0.5, 0.5, 0.5), reflectance_texture=1, normal_texture=2)]
    inst = [(0, 0, IDENTITY)]
    for i in range(32):
        r = rng.uniform(0.2, 0.6)
        c = (rng.uniform(-4, 4), rng.uniform(0.2, 2.0), rng.uniform(-4, 4))
        meshes.append(sphere_mesh(2, c, r))
        k = i % 6
        if k == 0:
            m = Material(MAT_DIFFUSE, reflectance=(0.5, 0.5, 0.5), reflectance_texture=3)
        elif k == 1:
            m = Material(MAT_DIFFUSE, reflectance=(0.5, 0.5, 0.5), reflectance_texture=4, normal_texture=7)
        elif k == 2:
            m = Material(MAT_METAL, reflectance=(1.0, 1.0, 1.0), roughness=0.3, eta=GOLD_ETA, k=GOLD_K,
                         roughness_texture=5)
        elif k == 3:
            m = Material(MAT_METAL, reflectance=(1.0, 1.0, 1.0), roughness=0.2, eta=GOLD_ETA, k=GOLD_K,
                         reflectance_texture=6, normal_texture=7)
        elif k == 4:
            m = Material(MAT_GLASS, roughness=0.15, interior_ior=1.5, normal_texture=7)
        else:
            m = _random_material(rng)
        mats.append(m)
        inst.append((len(meshes) - 1, len(mats) - 1, IDENTITY))
    lobes = [(d, 2.0, 50.0) for d in random_upper_dirs(rng, 3)]
    dome = Emitter(EMIT_DOME, texels=hdri(256, 128, lobes, rng))
    cam = look_at_camera((0, 3, -10), (0, 0, 0), (0, 1, 0), 45.0, width, height)
    return Scene(width, height, meshes, inst, mats, [directional(), dome], cam, spp=16, max_depth=5, rr_start=3,
                 name="textured", textures=tex)


def config2(seed=0, width=1920, height=1080, terrain_n=1024, objects=512, hdri_size=(2048, 1024)):
    rng = np.random.default_rng(seed)
    meshes = [terrain_mesh(terrain_n, 40.0, 2.0, 5, seed + 101, y0=-1.0)]
    mats = [Material(MAT_DIFFUSE, reflectance=(0.45, 0.42, 0.38))]
    inst = [(0, 0, IDENTITY)]
    for i in range(objects):
        c = (rng.uniform(-30, 30), rng.uniform(0.5, 3.0), rng.uniform(-20, 40))
        if rng.random() < 0.5:
            meshes.append(sphere_mesh(4, c, rng.uniform(0.3, 1.2)))
        else:
            R = rng.uniform(0.4, 1.0)
            meshes.append(torus_mesh(50, 50, c, R, R * rng.uniform(0.2, 0.4)))
        mats.append(_random_material(rng))
        inst.append((len(meshes) - 1, len(mats) - 1, IDENTITY))
    w, h = hdri_size
    lobes = [(d, 2.0, 200.0) for d in random_upper_dirs(rng, 8)]
    dome = Emitter(EMIT_DOME, texels=hdri(w, h, lobes, rng))
    cam = look_at_camera((0, 3, -10), (0, 0, 0), (0, 1, 0), 45.0, width, height)
    return Scene(width, height, meshes, inst, mats, [directional(), dome], cam, spp=64, max_depth=8, rr_start=3,
                 name="cfg2")


def config3(seed=0):
    s = config1(seed, 1920, 1080)
    s.spp, s.name = 128, "cfg3"
    return s


def config4(seed=0):
    rng = np.random.default_rng(seed + 7)
    lobe = [(random_upper_dirs(rng, 1)[0], 0.5, 5000.0)]
    dome = Emitter(EMIT_DOME, texels=hdri(2048, 1024, lobe, rng))
    s = config1(seed, 1920, 1080, glass_frac=0.6, glass_alpha=(0.01, 0.1), dome=dome)
    s.spp, s.max_depth, s.name = 128, 16, "cfg4"
    return s


def _rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([[a*a+b*b-c*c-d*d, 2*(b*c-a*d), 2*(b*d+a*c)],
                     [2*(b*c+a*d), a*a-b*b+c*c-d*d, 2*(c*d-a*b)],
                     [2*(b*d-a*c), 2*(c*d+a*b), a*a-b*b-c*c+d*d]])


def config5(seed=0, width=3840, height=2160, terrain_n=2048, unique=128, copies=12):
    rng = np.random.default_rng(seed)
    meshes = [terrain_mesh(terrain_n, 60.0, 2.5, 5, seed + 202, y0=-1.0)]
    mats = [Material(MAT_DIFFUSE, reflectance=(0.45, 0.42, 0.38))]
    inst = [(0, 0, IDENTITY)]
    for u in range(unique):
        if u % 2 == 0:
            meshes.append(sphere_mesh(4, (0, 0, 0), 0.6))       # 5,120 tris
        else:
            meshes.append(torus_mesh(44, 44, (0, 0, 0), 0.6, 0.2))  # 3,872 tris
        mats.append(_random_material(rng))
        for c in range(copies):
            s = rng.uniform(0.5, 2.0)
            L = _rotation(rng) * s
            t = (rng.uniform(-50, 50), rng.uniform(0.5, 4.0), rng.uniform(-30, 60))
            M = np.concatenate([L, np.asarray(t)[:, None]], 1).reshape(-1)
            inst.append((len(meshes) - 1, len(mats) - 1, tuple(float(x) for x in M)))
    lobes = [(d, 2.0, 200.0) for d in random_upper_dirs(rng, 8)]
    dome = Emitter(EMIT_DOME, texels=hdri(4096, 2048, lobes, rng))
    cam = look_at_camera((0, 3, -10), (0, 0, 0), (0, 1, 0), 45.0, width, height)
    return Scene(width, height, meshes, inst, mats, [directional(), dome], cam, spp=256, max_depth=16, rr_start=3,
                 name="cfg5")


CONFIGS = {1: config1, 2: config2, 3: config3, 4: config4, 5: config5}


def save_obj(path, meshes):
    """Writes meshes as one Wavefront OBJ file (one `o` group per mesh, v/vt/vn
    per corner; vt stores 1 - v so that the loader's v flip restores the uvs;
    positions with 9 significant digits, exact for float32)."""
    lines, base = [], 0
    for i, m in enumerate(meshes):
        lines.append(f"o mesh{i}")
        lines += [f"v {x:.9g} {y:.9g} {z:.9g}" for x, y, z in m.positions.astype(np.float32)]
        if m.uvs is not None:
            lines += [f"vt {float(u):.17g} {1.0 - float(v):.17g}" for u, v in m.uvs.astype(np.float32)]
        if m.normals is not None:
            lines += [f"vn {x:.9g} {y:.9g} {z:.9g}" for x, y, z in m.normals.astype(np.float32)]
        for tri in m.indices.astype(np.int64) + base + 1:
            if m.uvs is not None and m.normals is not None:
                lines.append("f " + " ".join(f"{k}/{k}/{k}" for k in tri))
            elif m.normals is not None:
                lines.append("f " + " ".join(f"{k}//{k}" for k in tri))
            elif m.uvs is not None:
                lines.append("f " + " ".join(f"{k}/{k}" for k in tri))
            else:
                lines.append("f " + " ".join(str(k) for k in tri))
        base += len(m.positions)
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")

