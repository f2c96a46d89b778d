"""colvillea_b200: a B200 (sm_100a) wavefront path tracer behind Colvillea's
integrator interface.

The Python layer mirrors `colvillea::core::Integrator`
(include/colvillea/librender/integrator.h:34-103): same method names and
meaning, errors raised as ClError instead of the reference's exit(-1).
All work runs in libcolvillea_b200.so (CUDA kernels for sm_100a, C ABI in
include/colvillea_b200.h); there is no CPU fallback.
"""
import ctypes
import enum

import numpy as np

from . import _native as N
from ._native import ClError

__all__ = ["IntegratorType", "Integrator", "RenderConfig", "ClError", "COMPAT_ALL", "DOME_ALIAS", "FILM_FP64",
           "PROFILE_STAGES", "TRACE_STATS", "TWO_LEVEL", "load_scene", "GuideConfig", "Guide", "RadianceCacheConfig", "Cache",
           "load_obj", "load_hdr", "write_pfm", "read_pfm"]

COMPAT_PDF, COMPAT_FRAME, COMPAT_ESCAPE, COMPAT_ALL = N.CL_COMPAT_PDF, N.CL_COMPAT_FRAME, N.CL_COMPAT_ESCAPE, N.CL_COMPAT_ALL
DOME_ALIAS, FILM_FP64, PROFILE_STAGES, TRACE_STATS = N.CL_DOME_ALIAS, N.CL_FILM_FP64, N.CL_PROFILE_STAGES, N.CL_TRACE_STATS
TWO_LEVEL = N.CL_TWO_LEVEL


class IntegratorType(enum.IntEnum):
    """IntegratorType (integrator.h:22-32)."""
    WavefrontDirectLighting = N.CL_INTEGRATOR_DIRECT_LIGHTING
    WavefrontPathTracing = N.CL_INTEGRATOR_PATH_TRACING


def RenderConfig(max_depth=5, rr_start_depth=0, flags=COMPAT_ALL, path_slots=0):
    return N.RenderConfig(max_depth, rr_start_depth, flags, path_slots)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


class Integrator:
    """A wavefront integrator on the current CUDA device (one stream)."""

    def __init__(self, handle, itype, width, height):
        self._h = handle
        self.type = itype
        self._size = (width, height)

    @staticmethod
    def createIntegrator(itype, width, height, config=None):
        """Integrator::createIntegrator (src/core/librender/integrator.cpp:10-22)."""
        h = ctypes.c_void_p()
        cfg = config if config is not None else RenderConfig()
        N.call("cl_integrator_create", int(itype), width, height, ctypes.byref(cfg), ctypes.byref(h))
        return Integrator(h, IntegratorType(itype), width, height)

    def close(self):
        if getattr(self, "_h", None):
            N.lib().cl_integrator_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # --- scene building (Integrator::build*) ---------------------------------
    def buildBLAS(self, meshes):
        """meshes: list of scenes.Mesh (positions, normals, tangents, uvs, indices)."""
        keep, descs = [], (N.MeshDesc * len(meshes))()
        for i, m in enumerate(meshes):
            arrs = [_f32(m.positions), None if m.normals is None else _f32(m.normals), _f32(m.tangents),
                    None if m.uvs is None else _f32(m.uvs), np.ascontiguousarray(m.indices, np.uint32)]
            keep.append(arrs)
            p, n, t, uv, idx = arrs
            descs[i] = N.MeshDesc(_ptr(p), _ptr(n), _ptr(t), _ptr(uv), len(p), _ptr(idx), len(idx))
        N.call("cl_build_meshes", self._h, descs, len(meshes))

    def buildTLAS(self, instances):
        """instances: list of (mesh_id, material_index, 3x4 row-major transform);
        covers buildTLAS and buildGeometryEntities (integrator.h:49-54)."""
        descs = (N.InstanceDesc * len(instances))()
        for i, (mid, mat, xf) in enumerate(instances):
            descs[i] = N.InstanceDesc(mid, mat, (ctypes.c_float * 12)(*xf))
        N.call("cl_build_instances", self._h, descs, len(instances))

    BVH_UPDATE = {"auto": N.CL_BVH_UPDATE_AUTO, "refit": N.CL_BVH_UPDATE_REFIT, "rebuild": N.CL_BVH_UPDATE_REBUILD}

    def updateVertices(self, mesh_id, positions, normals=None, tangents=None, bvh="auto"):
        """Shape edit (TriangleMesh::updateVertices, trianglemesh.h:111-118, then
        RenderEngine::compileAccelStructs): new vertex positions for mesh `mesh_id`
        (same count and triangles); the BVH is refitted ("refit"), rebuilt
        ("rebuild") or refitted and rebuilt if its surface-area cost grew past
        1.5x the built tree's ("auto"); the progressive iteration restarts."""
        p = _f32(positions)
        n = None if normals is None else _f32(normals)
        t = None if tangents is None else _f32(tangents)
        N.call("cl_update_mesh_vertices", self._h, mesh_id, _ptr(p), _ptr(n), _ptr(t), len(p), self.BVH_UPDATE[bvh])

    def bvh(self):
        """(nodes (n, 20) uint32, triangles (t, 12) float32): the built 8-wide BVH."""
        s = self.stats()
        nodes = np.empty((s["bvh_nodes"], 20), np.uint32)
        tris = np.empty((s["triangles"], 12), np.float32)
        N.call("cl_get_bvh", self._h, _ptr(nodes), nodes.nbytes, _ptr(tris), tris.nbytes)
        return nodes, tris

    def buildMaterials(self, materials):
        """scenes.Material list; texture fields are 1-based indices into the
        last buildTextures list (0 = none)."""
        descs = (N.MaterialDesc * len(materials))()
        for i, m in enumerate(materials):
            descs[i] = N.MaterialDesc(m.type, (ctypes.c_float * 3)(*m.reflectance), m.roughness, m.interior_ior,
                                      (ctypes.c_float * 3)(*m.eta), (ctypes.c_float * 3)(*m.k),
                                      getattr(m, "reflectance_texture", 0), getattr(m, "roughness_texture", 0),
                                      getattr(m, "normal_texture", 0))
        N.call("cl_build_materials", self._h, descs, len(materials))

    def buildTextures(self, textures):
        """scenes.Texture list (image textures: bilinear, wrap, sRGB decode for
        sRGB RGBA8)."""
        keep, descs = [], (N.TextureDesc * max(1, len(textures)))()
        for i, t in enumerate(textures):
            d, keep_arr = texture_desc(t)
            keep.append(keep_arr)
            descs[i] = d
        N.call("cl_build_textures", self._h, descs, len(textures))

    def buildEmitters(self, emitters):
        keep, descs = [], (N.EmitterDesc * len(emitters))()
        for i, e in enumerate(emitters):
            tex = None if e.texels is None else _f32(e.texels)
            keep.append(tex)
            h, w = (tex.shape[:2] if tex is not None else (0, 0))
            descs[i] = N.EmitterDesc(e.type, (ctypes.c_float * 3)(*e.intensity), (ctypes.c_float * 3)(*e.direction),
                                     e.angular_radius, _ptr(tex), w, h)
        N.call("cl_build_emitters", self._h, descs, len(emitters))

    def updateCamera(self, cam12):
        c = _f32(cam12)
        N.call("cl_update_camera", self._h, ctypes.byref(N.Camera(*(
            (ctypes.c_float * 3)(*c[3 * i:3 * i + 3]) for i in range(4)))))

    # --- rendering ------------------------------------------------------------
    def render(self, spp=1):
        """`spp` progressive iterations (Integrator::render, one per call in the reference)."""
        N.call("cl_render", self._h, spp)

    def resize(self, width, height):
        N.call("cl_resize", self._h, width, height)
        self._size = (width, height)

    def getFilmSize(self):
        w, h = ctypes.c_uint32(), ctypes.c_uint32()
        N.call("cl_get_film_size", self._h, ctypes.byref(w), ctypes.byref(h))
        return w.value, h.value

    def setIterationIndex(self, iteration):
        """Clear the film and continue from progressive frame `iteration`."""
        N.call("cl_set_iteration", self._h, int(iteration))

    def resetIterationIndex(self):
        N.call("cl_reset_iteration", self._h)

    def readbackFramebuffer(self, out=None):
        """Linear HDR mean radiance, (H, W, 4) float32."""
        w, h = self._size
        if out is None:
            out = np.empty((h, w, 4), np.float32)
        N.call("cl_readback_film", self._h, _ptr(out), out.nbytes)
        return out

    def readbackFramebufferAsync(self, out):
        """Queues the readback of the mean radiance into `out` ((H, W, 4) float32,
        best in page-locked memory) and returns; the copy overlaps the next
        render.  `out` is complete after readbackWait()."""
        w, h = self._size
        if out.shape != (h, w, 4) or out.dtype != np.float32 or not out.flags.c_contiguous:
            raise ValueError(f"out must be a contiguous ({h}, {w}, 4) float32 array")
        N.call("cl_readback_film_async", self._h, _ptr(out), out.nbytes)
        self._pending = out
        return out

    def readbackWait(self):
        N.call("cl_readback_wait", self._h)
        self._pending = None

    def readbackFilmStats(self):
        """FP64 per-pixel (sum, sumsq) of per-sample radiance, each (H*W, 3)."""
        w, h = self._size
        s1 = np.zeros((w * h, 3)); s2 = np.zeros((w * h, 3))
        N.call("cl_readback_film_stats", self._h, _ptr(s1), _ptr(s2), s1.size)
        return s1, s2

    def stats(self):
        s = N.Stats()
        N.call("cl_get_stats", self._h, ctypes.byref(s))
        return s.as_dict()

    # --- ray queries ------------------------------------------------------------
    def traceRays(self, rays):
        rays = _f32(rays)
        n = len(rays)
        t = np.zeros(n, np.float32); prim = np.zeros(n, np.uint32)
        b1 = np.zeros(n, np.float32); b2 = np.zeros(n, np.float32)
        N.call("cl_trace_rays", self._h, _ptr(rays), n, _ptr(t), _ptr(prim), _ptr(b1), _ptr(b2))
        return t, prim, b1, b2

    def occludedRays(self, rays):
        rays = _f32(rays)
        occ = np.zeros(len(rays), np.uint8)
        N.call("cl_occluded_rays", self._h, _ptr(rays), len(rays), _ptr(occ))
        return occ

    def traceStats(self, rays):
        rays = _f32(rays)
        a, b = ctypes.c_uint64(), ctypes.c_uint64()
        N.call("cl_trace_stats", self._h, _ptr(rays), len(rays), ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def domeTables(self, w, h):
        pU = np.zeros((w + 1) * h, np.float32); cU = np.zeros_like(pU)
        pV = np.zeros(h + 1, np.float32); cV = np.zeros_like(pV)
        N.call("cl_get_dome_tables", self._h, _ptr(pU), _ptr(cU), _ptr(pV), _ptr(cV))
        return pU, cU, pV, cV

    def waveRays(self):
        """CL_PROFILE_STAGES: closest-hit rays of each wave of the last render."""
        buf = np.zeros(256, np.uint64)
        n = ctypes.c_uint32()
        N.call("cl_get_wave_rays", self._h, _ptr(buf), len(buf), ctypes.byref(n))
        return [int(x) for x in buf[:min(n.value, len(buf))]]

    def domeAliasTables(self, w, h):
        row = np.zeros(2 * h, np.uint32); col = np.zeros(2 * w * h, np.uint32)
        N.call("cl_get_dome_alias_tables", self._h, _ptr(row), _ptr(col))
        return row, col

    def domeAliasSample(self, u2):
        u2 = _f32(u2)
        n = len(u2)
        d = np.zeros((n, 3), np.float32); p = np.zeros(n, np.float32); v = np.zeros((n, 3), np.float32)
        N.call("cl_dome_alias_sample", self._h, _ptr(u2), _ptr(d), _ptr(p), _ptr(v), n)
        return d, p, v


def GuideConfig(**kw):
    """cl_guide_config with the library's defaults, fields overridden by kw
    (resolutions: a sequence of 16 level resolutions)."""
    c = N.GuideConfig()
    N.lib().cl_guide_default_config(ctypes.byref(c))
    for k, v in kw.items():
        if k == "resolutions":
            for i, r in enumerate(v):
                c.resolutions[i] = int(r)
        else:
            setattr(c, k, v)
    return c


def default_resolutions(n_min, n_max):
    r = np.zeros(16, np.uint32)
    N.call("cl_guide_default_resolutions", float(n_min), float(n_max), _ptr(r))
    return r


class Guide:
    """The neural path-guiding network (no counterpart in the reference):
    hash grid + one-blob encoding, 96-64-64-64-64-48 MLP on the tensor cores,
    8-lobe vMF mixture head, Adam training."""

    def __init__(self, handle, owned=True):
        self._h = handle
        self._owned = owned

    @staticmethod
    def create(config=None):
        h = ctypes.c_void_p()
        cfg = config if config is not None else GuideConfig()
        N.call("cl_guide_create", ctypes.byref(cfg), ctypes.byref(h))
        return Guide(h)

    def close(self):
        if getattr(self, "_h", None) and self._owned:
            N.lib().cl_guide_destroy(self._h)
        self._h = None

    def __del__(self):
        self.close()

    def param_count(self):
        n = ctypes.c_uint64()
        N.call("cl_guide_param_count", self._h, ctypes.byref(n))
        return n.value

    def resolutions(self):
        r = np.zeros(16, np.uint32)
        N.call("cl_guide_get_resolutions", self._h, _ptr(r))
        return r

    def get_params(self):
        p = np.zeros(self.param_count(), np.float32)
        N.call("cl_guide_get_params", self._h, _ptr(p), p.size)
        return p

    def set_params(self, p):
        p = _f32(p)
        N.call("cl_guide_set_params", self._h, _ptr(p), p.size)

    def forward(self, in9):
        in9 = _f32(in9)
        out = np.zeros((len(in9), 48), np.float32)
        N.call("cl_guide_forward", self._h, _ptr(in9), len(in9), _ptr(out))
        return out

    def gradient(self, rec14):
        """rec14 rows: position, normal, wo, omega, weight, BSDF pdf of omega."""
        rec14 = _f32(rec14)
        assert rec14.ndim == 2 and rec14.shape[1] == 14
        g = np.zeros(self.param_count(), np.float32)
        loss = ctypes.c_double()
        N.call("cl_guide_gradient", self._h, _ptr(rec14), len(rec14), ctypes.byref(loss), _ptr(g))
        return loss.value, g

    def train_step(self, rec14):
        rec14 = _f32(rec14)
        assert rec14.ndim == 2 and rec14.shape[1] == 14
        loss = ctypes.c_double()
        N.call("cl_guide_train_step", self._h, _ptr(rec14), len(rec14), ctypes.byref(loss))
        return loss.value

    def sample(self, in9, u3):
        in9, u3 = _f32(in9), _f32(u3)
        d = np.zeros((len(in9), 3), np.float32); p = np.zeros(len(in9), np.float32)
        N.call("cl_guide_sample", self._h, _ptr(in9), _ptr(u3), len(in9), _ptr(d), _ptr(p))
        return d, p

    def pdf(self, in9, dirs):
        in9, dirs = _f32(in9), _f32(dirs)
        p = np.zeros(len(in9), np.float32)
        N.call("cl_guide_pdf", self._h, _ptr(in9), _ptr(dirs), len(in9), _ptr(p))
        return p


def RadianceCacheConfig(**kw):
    """cl_radiance_cache_config with the library's defaults; `network` takes a
    dict of cl_guide_config fields (hash grid, Adam, batch)."""
    c = N.RadianceCacheConfig()
    N.lib().cl_radiance_cache_default_config(ctypes.byref(c))
    for k, v in kw.items():
        if k == "network":
            for nk, nv in v.items():
                if nk == "resolutions":
                    for i, r in enumerate(nv):
                        c.network.resolutions[i] = int(r)
                else:
                    setattr(c.network, nk, nv)
        else:
            setattr(c, k, v)
    return c


class Cache:
    """The neural radiance cache network (hash grid + one-blob encoding,
    96-64-64-16 MLP on the tensor cores, RGB in outputs 0-2)."""

    def __init__(self, handle, owned=True):
        self._h = handle
        self._owned = owned

    @staticmethod
    def create(network=None):
        h = ctypes.c_void_p()
        cfg = network if network is not None else RadianceCacheConfig().network
        N.call("cl_cache_create", ctypes.byref(cfg), ctypes.byref(h))
        return Cache(h)

    def close(self):
        if getattr(self, "_h", None) and self._owned:
            N.lib().cl_cache_destroy(self._h)
        self._h = None

    def __del__(self):
        self.close()

    def param_count(self):
        n = ctypes.c_uint64()
        N.call("cl_cache_param_count", self._h, ctypes.byref(n))
        return n.value

    def resolutions(self):
        r = np.zeros(16, np.uint32)
        N.call("cl_cache_get_resolutions", self._h, _ptr(r))
        return r

    def get_params(self):
        p = np.zeros(self.param_count(), np.float32)
        N.call("cl_cache_get_params", self._h, _ptr(p), p.size)
        return p

    def set_params(self, p):
        p = _f32(p)
        N.call("cl_cache_set_params", self._h, _ptr(p), p.size)

    def forward(self, in9):
        in9 = _f32(in9)
        out = np.zeros((len(in9), 16), np.float32)
        N.call("cl_cache_forward", self._h, _ptr(in9), len(in9), _ptr(out))
        return out

    def gradient(self, rec12):
        """rec12 rows: position, normal, wo, target RGB."""
        rec12 = _f32(rec12)
        assert rec12.ndim == 2 and rec12.shape[1] == 12
        g = np.zeros(self.param_count(), np.float32)
        loss = ctypes.c_double()
        N.call("cl_cache_gradient", self._h, _ptr(rec12), len(rec12), ctypes.byref(loss), _ptr(g))
        return loss.value, g

    def train_step(self, rec12):
        rec12 = _f32(rec12)
        assert rec12.ndim == 2 and rec12.shape[1] == 12
        loss = ctypes.c_double()
        N.call("cl_cache_train_step", self._h, _ptr(rec12), len(rec12), ctypes.byref(loss))
        return loss.value


def _set_radiance_cache(self, config):
    """Path tracing with the neural radiance cache (None: off)."""
    N.call("cl_integrator_set_radiance_cache", self._h, ctypes.byref(config) if config is not None else None)


def _cache(self):
    h = ctypes.c_void_p()
    N.call("cl_integrator_get_cache", self._h, ctypes.byref(h))
    return Cache(h, owned=False) if h.value else None


def _cache_stats(self):
    s = N.GuideStats()
    N.call("cl_integrator_cache_stats", self._h, ctypes.byref(s))
    return s.as_dict()


Integrator.setRadianceCache = _set_radiance_cache
Integrator.cache = _cache
Integrator.cacheStats = _cache_stats


def _set_guiding(self, config):
    """Guided path tracing with a fresh network (None: off)."""
    N.call("cl_integrator_set_guiding", self._h, ctypes.byref(config) if config is not None else None)


def _guide(self):
    h = ctypes.c_void_p()
    N.call("cl_integrator_get_guide", self._h, ctypes.byref(h))
    return Guide(h, owned=False) if h.value else None


def _guide_stats(self):
    s = N.GuideStats()
    N.call("cl_integrator_guide_stats", self._h, ctypes.byref(s))
    return s.as_dict()


def _guide_probe(self, capacity):
    """First-wave rows of the fused guide inference: (n, 52) float32 per
    guided ray {in9, ray index bits, 8 x (mu, kappa), 8 weights, pad}."""
    rows = np.zeros((max(int(capacity), 1), 52), np.float32)
    n = ctypes.c_uint32()
    N.call("cl_integrator_guide_probe", self._h, int(capacity), _ptr(rows), ctypes.byref(n))
    return rows[:n.value]


Integrator.setGuiding = _set_guiding
Integrator.guide = _guide
Integrator.guideStats = _guide_stats
Integrator.guideProbe = _guide_probe


# --- scene ingestion and film output (MeshImporter / ImageUtils, src/delegate) ---
def texture_desc(t):
    """(TextureDesc, array to keep alive) for a scenes.Texture."""
    a = np.ascontiguousarray(t.texels)
    if a.ndim != 3 or a.shape[2] != 4 or a.dtype not in (np.uint8, np.float32):
        raise ValueError("texture texels must be (h, w, 4) uint8 or float32")
    fmt = N.CL_TEXTURE_RGBA8 if a.dtype == np.uint8 else N.CL_TEXTURE_RGBA32F
    return N.TextureDesc(fmt, a.shape[1], a.shape[0], int(bool(t.srgb)), _ptr(a)), a


def texture_lookup(t, uv):
    """RGBA lookups in one texture, set up like the integrator's (texture unit)."""
    d, a = texture_desc(t)
    uv = _f32(uv).reshape(-1, 2)
    out = np.zeros((len(uv), 4), np.float32)
    N.call("cl_unit_texture_lookup", ctypes.byref(d), _ptr(uv), _ptr(out), len(uv))
    return out


def normal_frame(inputs16):
    """cl_unit_normal_frame: (n, 16) {wo, dpdu, dpdv, base normal, texel rgb, pull-up} -> (n, 3, 3) {s, t, n}."""
    x = _f32(inputs16).reshape(-1, 16)
    out = np.zeros((len(x), 9), np.float32)
    N.call("cl_unit_normal_frame", _ptr(x), _ptr(out), len(x))
    return out.reshape(-1, 3, 3)


def tc_wait_timeout():
    """cl_unit_tc_wait_timeout: the network kernels' bounded tensor-core wait on a
    barrier that nothing arrives at.  Returns (status, seconds waited); the
    expected status is CL_ERR_TIMEOUT after about one second."""
    ns = ctypes.c_uint64(0)
    st = N.lib().cl_unit_tc_wait_timeout(ctypes.byref(ns))
    return int(st), ns.value * 1e-9


def load_obj(path):
    """Meshes of a Wavefront OBJ file (one per o/g/usemtl group) as
    scenes.Mesh: triangulated, unified vertices, normals (smooth where the
    file has none), uvs with v flipped, tangents from the uvs."""
    from .scenes import Mesh
    h = ctypes.c_void_p()
    N.call("cl_obj_load", str(path).encode(), ctypes.byref(h))
    try:
        n = ctypes.c_uint32()
        N.call("cl_obj_mesh_count", h, ctypes.byref(n))
        out = []
        for i in range(n.value):
            d = N.MeshDesc()
            N.call("cl_obj_get_mesh", h, i, ctypes.byref(d))
            nv, nt = d.num_vertices, d.num_triangles

            def arr(ptr, k, dt=np.float32, ct=ctypes.c_float):
                if not ptr:
                    return None
                return np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ct)), shape=(k,)).astype(dt).copy()
            pos = arr(d.positions, 3 * nv).reshape(nv, 3)
            nrm = arr(d.normals, 3 * nv).reshape(nv, 3)
            tan = arr(d.tangents, 3 * nv).reshape(nv, 3)
            uv = arr(d.uvs, 2 * nv)
            idx = arr(d.indices, 3 * nt, np.uint32, ctypes.c_uint32).reshape(nt, 3)
            out.append(Mesh(pos, nrm, tan, None if uv is None else uv.reshape(nv, 2), idx))
        return out
    finally:
        N.lib().cl_obj_free(h)


def _take_image(ptr, w, h):
    try:
        return np.ctypeslib.as_array(ptr, shape=(h.value * w.value * 4,)).reshape(h.value, w.value, 4).copy()
    finally:
        N.lib().cl_image_free(ptr)


def load_hdr(path):
    """Radiance .hdr image as (h, w, 4) float32 (alpha 1), rows top to bottom."""
    ptr, w, h = ctypes.POINTER(ctypes.c_float)(), ctypes.c_uint32(), ctypes.c_uint32()
    N.call("cl_image_load_hdr", str(path).encode(), ctypes.byref(ptr), ctypes.byref(w), ctypes.byref(h))
    return _take_image(ptr, w, h)


def write_pfm(path, rgba):
    """Writes an (h, w, 4) (or (h, w, 3)) float image, e.g. readbackFramebuffer(), as PFM."""
    img = np.asarray(rgba, np.float32)
    if img.shape[-1] == 3:
        img = np.concatenate([img, np.ones(img.shape[:2] + (1,), np.float32)], -1)
    img = np.ascontiguousarray(img)
    N.call("cl_image_write_pfm", str(path).encode(), _ptr(img), img.shape[1], img.shape[0])


def read_pfm(path):
    ptr, w, h = ctypes.POINTER(ctypes.c_float)(), ctypes.c_uint32(), ctypes.c_uint32()
    N.call("cl_image_read_pfm", str(path).encode(), ctypes.byref(ptr), ctypes.byref(w), ctypes.byref(h))
    return _take_image(ptr, w, h)


def load_scene(scene, itype=IntegratorType.WavefrontPathTracing, flags=COMPAT_ALL, max_depth=None, rr_start=None,
               path_slots=0):
    """Integrator for a colvillea_b200.scenes.Scene, scene built, camera set
    (the RenderEngine::startRendering compile sequence, renderengine.cpp:27-114)."""
    cfg = RenderConfig(scene.max_depth if max_depth is None else max_depth,
                       scene.rr_start if rr_start is None else rr_start, flags, path_slots)
    it = Integrator.createIntegrator(itype, scene.width, scene.height, cfg)
    try:
        if getattr(scene, "textures", None):
            it.buildTextures(scene.textures)
        it.buildMaterials(scene.materials)
        it.buildBLAS(scene.meshes)
        it.buildTLAS(scene.instances)
        it.buildEmitters(scene.emitters)
        it.updateCamera(scene.camera)
    except BaseException:
        it.close()  # a refused build step must not leave the integrator's device memory behind
        raise
    return it
