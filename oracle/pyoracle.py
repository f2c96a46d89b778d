"""ORACLE — test infrastructure only.

ctypes bindings for oracle/liboracle.so, the CPU restatement of the
reference's path-tracing arithmetic (oracle/orc_core.h, orc_emit.h,
oracle.cpp).  Only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline use it, as the checker.  Nothing in colvillea_b200 imports it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

COMPAT_PDF = 1 << 0
COMPAT_FRAME = 1 << 1
COMPAT_ESCAPE = 1 << 2
COMPAT_ALL = COMPAT_PDF | COMPAT_FRAME | COMPAT_ESCAPE
DOME_ALIAS = 1 << 4
DIRECT_LIGHTING = 1 << 8

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.orc_scene_create.restype = ctypes.c_void_p
        _lib.orc_scene_create.argtypes = [ctypes.c_void_p]
        _lib.orc_scene_destroy.argtypes = [ctypes.c_void_p]
        _lib.orc_scene_bvh_nodes.restype = ctypes.c_uint32
        _lib.orc_scene_bvh_nodes.argtypes = [ctypes.c_void_p]
    return _lib


def P(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


class OrcSceneDesc(ctypes.Structure):
    _fields_ = [
        ("pos", ctypes.c_void_p), ("nrm", ctypes.c_void_p), ("tan", ctypes.c_void_p), ("uv", ctypes.c_void_p),
        ("nverts", ctypes.c_uint32), ("idx", ctypes.c_void_p), ("tri_material", ctypes.c_void_p),
        ("ntris", ctypes.c_uint32), ("materials", ctypes.c_void_p), ("nmaterials", ctypes.c_uint32),
        ("emitters", ctypes.c_void_p), ("nemitters", ctypes.c_uint32), ("dome_texels", ctypes.c_void_p),
        ("camera", ctypes.c_void_p), ("textures", ctypes.c_void_p), ("ntextures", ctypes.c_uint32),
    ]


class OrcTexture(ctypes.Structure):
    _fields_ = [("format", ctypes.c_int), ("w", ctypes.c_int), ("h", ctypes.c_int), ("srgb", ctypes.c_int),
                ("texels", ctypes.c_void_p)]


def orc_texture(t):
    """(OrcTexture, array to keep alive) for a scenes.Texture."""
    a = np.ascontiguousarray(t.texels)
    fmt = 0 if a.dtype == np.uint8 else 1
    if fmt == 1:
        a = np.ascontiguousarray(a, np.float32)
    return OrcTexture(fmt, a.shape[1], a.shape[0], int(bool(t.srgb)), P(a)), a


class OrcConfig(ctypes.Structure):
    _fields_ = [("max_depth", ctypes.c_uint32), ("rr_start_depth", ctypes.c_uint32), ("flags", ctypes.c_uint32),
                ("frame0", ctypes.c_uint32)]


class OracleScene:
    """A flattened scene (see colvillea_b200.scenes.FlatScene) with its CPU BVH."""

    def __init__(self, flat):
        self._keep = [f32(flat.pos), f32(flat.nrm), f32(flat.tan), f32(flat.uv), u32(flat.idx), u32(flat.tri_material),
                      f32(flat.materials), f32(flat.emitters), f32(flat.dome_texels), f32(flat.camera)]
        pos, nrm, tan, uv, idx, tm, mats, ems, dome, cam = self._keep
        texs = getattr(flat, "textures", None) or []
        tarr = (OrcTexture * max(1, len(texs)))()
        for i, t in enumerate(texs):
            tarr[i], a = orc_texture(t)
            self._keep.append(a)
        self._keep.append(tarr)
        d = OrcSceneDesc(P(pos), P(nrm), P(tan), P(uv), len(pos), P(idx), P(tm), len(idx), P(mats), len(mats),
                         P(ems), len(ems), P(dome), P(cam), ctypes.cast(tarr, ctypes.c_void_p), len(texs))
        self.h = lib().orc_scene_create(ctypes.byref(d))
        self.width, self.height = flat.width, flat.height
        self.ntris = len(idx)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_scene_destroy(self.h)
            self.h = None

    def bvh_nodes(self):
        return lib().orc_scene_bvh_nodes(self.h)

    def trace(self, rays, bruteforce=False, threads=8):
        rays = f32(rays)
        n = len(rays)
        t = np.zeros(n, np.float32); i = np.zeros(n, np.uint32)
        b1 = np.zeros(n, np.float32); b2 = np.zeros(n, np.float32)
        lib().orc_trace(ctypes.c_void_p(self.h), P(rays), ctypes.c_uint32(n), ctypes.c_int(int(bruteforce)), P(t), P(i),
                        P(b1), P(b2), ctypes.c_int(threads))
        return t, i, b1, b2

    def occluded(self, rays, threads=8):
        rays = f32(rays)
        occ = np.zeros(len(rays), np.uint8)
        lib().orc_occluded(ctypes.c_void_p(self.h), P(rays), ctypes.c_uint32(len(rays)), P(occ), ctypes.c_int(threads))
        return occ

    def dome_tables(self, w, h):
        pU = np.zeros((w + 1) * h, np.float32); cU = np.zeros_like(pU)
        pV = np.zeros(h + 1, np.float32); cV = np.zeros_like(pV)
        lib().orc_scene_dome_tables(ctypes.c_void_p(self.h), P(pU), P(cU), P(pV), P(cV))
        return pU, cU, pV, cV

    def set_dome_tables(self, tables, alias=None):
        """Use given dome tables (pU, cU, pV, cV) and, for DOME_ALIAS
        renders, alias tables (row, col as uint32 pairs) instead of the
        oracle's own FP32-built ones."""
        pU, cU, pV, cV = (f32(t) for t in tables)
        row, col = (u32(alias[0]), u32(alias[1])) if alias is not None else (None, None)
        self._keep += [pU, cU, pV, cV, row, col]
        r = lib().orc_scene_set_dome_tables(ctypes.c_void_p(self.h), P(pU), P(cU), P(pV), P(cV), P(row), P(col))
        assert r == 0, "scene has no dome"

    def render(self, spp, max_depth=5, rr_start=0, flags=COMPAT_ALL, frame0=0, pixels=None, threads=8):
        """Returns (sum, sumsq) FP64 arrays of shape (npix, 3) and ray counters."""
        W, H = self.width, self.height
        pix = u32(pixels) if pixels is not None else None
        n = len(pix) if pix is not None else W * H
        s1 = np.zeros((n, 3), np.float64); s2 = np.zeros((n, 3), np.float64)
        cnt = np.zeros(2, np.uint64)
        cfg = OrcConfig(max_depth, rr_start, flags, frame0)
        lib().orc_render(ctypes.c_void_p(self.h), ctypes.byref(cfg), ctypes.c_uint32(W), ctypes.c_uint32(H),
                         ctypes.c_uint32(spp), P(pix), ctypes.c_uint32(n), P(s1), P(s2), ctypes.c_int(threads), P(cnt))
        return s1, s2, cnt


# --- unit functions ---------------------------------------------------------
def bsdf_eval(btype, params, wo, wi, fp64=False):
    params, wo, wi = f32(params), f32(wo), f32(wi)
    n = len(wo)
    out = np.zeros((n, 3), np.float32); out64 = np.zeros((n, 3), np.float64)
    lib().orc_bsdf_eval(btype, P(params), P(wo), P(wi), P(out), n, int(fp64), P(out64))
    return out64 if fp64 else out


def bsdf_pdf(btype, params, wo, wi, compat=True, fp64=False):
    params, wo, wi = f32(params), f32(wo), f32(wi)
    n = len(wo)
    out = np.zeros(n, np.float32); out64 = np.zeros(n, np.float64)
    lib().orc_bsdf_pdf(btype, P(params), P(wo), P(wi), P(out), n, int(compat), int(fp64), P(out64))
    return out64 if fp64 else out


def bsdf_sample(btype, params, wo, u2, fp64=False):
    params, wo, u2 = f32(params), f32(wo), f32(u2)
    n = len(wo)
    wi = np.zeros((n, 3), np.float32); pdf = np.zeros(n, np.float32); val = np.zeros((n, 3), np.float32)
    wi64 = np.zeros((n, 3)); pdf64 = np.zeros(n); val64 = np.zeros((n, 3))
    lib().orc_bsdf_sample(btype, P(params), P(wo), P(u2), P(wi), P(pdf), P(val), n, int(fp64), P(wi64), P(pdf64),
                          P(val64))
    return (wi64, pdf64, val64) if fp64 else (wi, pdf, val)


def ggx_eval(alpha, m, wi, wo):
    alpha, m, wi, wo = f32(alpha), f32(m), f32(wi), f32(wo)
    n = len(alpha)
    D, G1, G, pa = (np.zeros(n, np.float32) for _ in range(4))
    lib().orc_ggx_eval(P(alpha), P(m), P(wi), P(wo), P(D), P(G1), P(G), P(pa), n)
    return D, G1, G, pa


def ggx_sample(alpha, u2):
    alpha, u2 = f32(alpha), f32(u2)
    n = len(alpha)
    m = np.zeros((n, 3), np.float32); pdf = np.zeros(n, np.float32)
    lib().orc_ggx_sample(P(alpha), P(u2), P(m), P(pdf), n)
    return m, pdf


def fresnel_conductor(cosi, eta, k):
    cosi, eta, k = f32(cosi), f32(eta), f32(k)
    out = np.zeros((len(cosi), 3), np.float32)
    lib().orc_fresnel_conductor(P(cosi), P(eta), P(k), P(out), len(cosi))
    return out


def fresnel_dielectric(cosi, eta):
    cosi, eta = f32(cosi), f32(eta)
    F = np.zeros(len(cosi), np.float32); ct = np.zeros(len(cosi), np.float32)
    lib().orc_fresnel_dielectric(P(cosi), P(eta), P(F), P(ct), len(cosi))
    return F, ct


def warp(u2):
    u2 = f32(u2)
    n = len(u2)
    d = np.zeros((n, 2), np.float32); h = np.zeros((n, 3), np.float32)
    lib().orc_warp(P(u2), P(d), P(h), n)
    return d, h


def make_frame(a):
    a = f32(a)
    b = np.zeros_like(a); c = np.zeros_like(a)
    lib().orc_make_frame(P(a), P(b), P(c), len(a))
    return b, c


def frame(s, t, n, v):
    s, t, n, v = f32(s), f32(t), f32(n), f32(v)
    loc = np.zeros_like(v); wld = np.zeros_like(v)
    lib().orc_frame(P(s), P(t), P(n), P(v), P(loc), P(wld), len(v))
    return loc, wld


def texture_lookup(t, uv):
    """Texture-unit model (bilinear, 8-bit weights rounded half up, wrap; RGBA8 decoded first)."""
    d, a = orc_texture(t)
    uv = f32(uv).reshape(-1, 2)
    out = np.zeros((len(uv), 4), np.float32)
    lib().orc_texture_lookup(ctypes.byref(d), P(uv), P(out), len(uv))
    return out


def normal_frame(inputs16, fp64=False):
    """(n, 16) {wo, dpdu, dpdv, base normal, texel rgb, pull-up} -> (n, 3, 3) {s, t, n}."""
    x = f32(inputs16).reshape(-1, 16)
    out = np.zeros((len(x), 9), np.float32)
    lib().orc_normal_frame(P(x), P(out), len(x), int(fp64))
    return out.reshape(-1, 3, 3)


def pcg4d(v):
    v = u32(v)
    out = np.zeros_like(v)
    lib().orc_pcg4d(P(v), P(out), len(v))
    return out


def sampler_sequence(pxpyframe, m):
    p = u32(pxpyframe)
    out = np.zeros((len(p), m), np.float32)
    lib().orc_sampler_sequence(P(p), len(p), m, P(out))
    return out


def dome_build_tables(texels, w, h):
    texels = f32(texels)
    pU = np.zeros((w + 1) * h, np.float32); cU = np.zeros_like(pU)
    pV = np.zeros(h + 1, np.float32); cV = np.zeros_like(pV)
    lib().orc_dome_build_tables(P(texels), w, h, P(pU), P(cU), P(pV), P(cV))
    return pU, cU, pV, cV


def dome_sample(texels, w, h, tables, u2):
    texels, u2 = f32(texels), f32(u2)
    pU, cU, pV, cV = (f32(t) for t in tables)
    n = len(u2)
    d = np.zeros((n, 3), np.float32); pdf = np.zeros(n, np.float32); val = np.zeros((n, 3), np.float32)
    lib().orc_dome_sample(P(texels), w, h, P(pU), P(cU), P(pV), P(cV), P(u2), P(d), P(pdf), P(val), n)
    return d, pdf, val


def dome_pdf_eval(texels, w, h, tables, dirs):
    texels, dirs = f32(texels), f32(dirs)
    pU, _, pV, _ = (f32(t) for t in tables)
    n = len(dirs)
    pdf = np.zeros(n, np.float32); val = np.zeros((n, 3), np.float32)
    lib().orc_dome_pdf_eval(P(texels), w, h, P(pU), P(pV), P(dirs), P(pdf), P(val), n)
    return pdf, val


def directional_sample(params7, u2):
    p, u2 = f32(params7), f32(u2)
    n = len(u2)
    d = np.zeros((n, 3), np.float32); pdf = np.zeros(n, np.float32); val = np.zeros((n, 3), np.float32)
    lib().orc_directional_sample(P(p), P(u2), P(d), P(pdf), P(val), n)
    return d, pdf, val


def hit_attributes(flat, prim, b1, b2):
    prim, b1, b2 = u32(prim), f32(b1), f32(b2)
    out = np.zeros((len(prim), 17), np.float32)
    keep = [f32(flat.pos), f32(flat.nrm), f32(flat.tan), f32(flat.uv), u32(flat.idx)]
    lib().orc_hit_attributes(*(P(k) for k in keep), P(prim), P(b1), P(b2), P(out), len(prim))
    return out
