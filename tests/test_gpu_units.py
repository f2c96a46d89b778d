"""GPU unit kernels (cl_unit_*: the integrator's device functions) against the
reference's own outputs (tests/golden, compiled from its sources) and the
oracle, within 4 ulp in FP32; rarer differences must be explained by the FP64
evaluation of the same formula (ill-conditioned spots, branch flips)."""
import numpy as np
import pytest

from colvillea_b200 import _native as N
from conftest import ulp_diff
from gpu_util import P, bilinear64, check_ulp, check_vec, f32, gpu_bsdf_eval, gpu_bsdf_pdf, gpu_bsdf_sample

pytestmark = pytest.mark.gpu
BSDFS = [(0, "diffuse"), (1, "conductor"), (2, "dielectric")]


def test_pcg4d_and_sampler_exact(native, golden, oracle):
    v = golden["pcg4d_in"]
    out = np.zeros_like(v)
    N.call("cl_unit_pcg4d", P(v), P(out), len(v))
    assert np.array_equal(out, golden["pcg4d_out"])
    s = golden["sampler_seeds"]
    m = golden["sampler_seq"].shape[1]
    seq = np.zeros((len(s), m), np.float32)
    N.call("cl_unit_sampler_sequence", P(s), len(s), m, P(seq))
    assert ulp_diff(seq, golden["sampler_seq"]).max() == 0


def check_sampling(name, btype, got, ref, ref64):
    """BSDF::sample outputs (wi, pdf, value).  They go through sinf/cosf
    (CUDA vs glibc, up to 2 ulp apart), amplified where the formula is
    ill-conditioned: at least 97% within 4 ulp, the rest explained by the FP64
    evaluation or, for the cosine-weighted diffuse pdf z / pi with
    z = sqrt(1 - r^2), by its relative condition r^2 / z^2."""
    cond = None
    if btype == 0:
        z = np.abs(np.asarray(ref[0], np.float64)[:, 2])
        cond = 4 + 4 * (1 - z * z) / np.maximum(z * z, 1e-12)
    check_vec(f"{name}.sample.wi", got[0], ref[0], ref64=ref64[0], min_frac=0.97, max_unexplained_frac=1e-3)
    check_ulp(f"{name}.sample.pdf", got[1], ref[1], ref64=ref64[1], min_frac=0.97, max_unexplained_frac=1e-3,
              cond_ulp=cond)
    check_vec(f"{name}.sample.value", got[2], ref[2], ref64=ref64[2], min_frac=0.97, max_unexplained_frac=1e-3)


@pytest.mark.parametrize("btype,name", BSDFS)
def test_bsdf_vs_reference_golden(native, golden, oracle, btype, name):
    g = lambda k: golden[f"{name}_{k}"]
    # eval and pdf: every value within 4 ulp of the reference's own code
    ev = gpu_bsdf_eval(btype, g("params"), g("wo"), g("wi"))
    check_ulp(f"{name}.eval", ev, g("eval"), min_frac=1.0)
    pdf = gpu_bsdf_pdf(btype, g("params"), g("wo"), g("wi"))
    check_ulp(f"{name}.pdf", pdf, g("pdf"), min_frac=1.0)
    # sampling goes through sinf/cosf (CUDA vs glibc): outliers explained by FP64
    wi, spdf, sval = gpu_bsdf_sample(btype, g("params"), g("wo"), g("u2"))
    wi64, spdf64, sval64 = oracle.bsdf_sample(btype, g("params"), g("wo"), g("u2"), fp64=True)
    check_sampling(name, btype, (wi, spdf, sval), (g("swi"), g("spdf"), g("sval")), (wi64, spdf64, sval64))


@pytest.mark.parametrize("btype,name", BSDFS)
def test_bsdf_vs_oracle_large(native, oracle, btype, name):
    """2^16 seeded cases per BSDF, reference (compat) and corrected pdfs."""
    rng = np.random.default_rng(100 + btype)
    n = 1 << 16
    p = np.zeros((n, 11), np.float32)
    p[:, 0:3] = rng.uniform(0, 1, (n, 3)); p[:, 3] = rng.uniform(0.002, 0.8, n); p[:, 4] = rng.uniform(1.05, 2.4, n)
    p[:, 5:8] = rng.uniform(0.05, 2.0, (n, 3)); p[:, 8:11] = rng.uniform(0.5, 5.0, (n, 3))
    wo = rng.normal(size=(n, 3)); wo /= np.linalg.norm(wo, axis=1, keepdims=True)
    wi = rng.normal(size=(n, 3)); wi /= np.linalg.norm(wi, axis=1, keepdims=True)
    wo[: n // 2, 2] = np.abs(wo[: n // 2, 2]); wi[: n // 2, 2] = np.abs(wi[: n // 2, 2])
    u2 = rng.uniform(0, 1, (n, 2)).astype(np.float32)
    wo, wi = f32(wo), f32(wi)
    check_ulp(f"{name}.eval[64k]", gpu_bsdf_eval(btype, p, wo, wi), oracle.bsdf_eval(btype, p, wo, wi), min_frac=1.0)
    for compat in (True, False):
        check_ulp(f"{name}.pdf[64k,compat={compat}]", gpu_bsdf_pdf(btype, p, wo, wi, compat),
                  oracle.bsdf_pdf(btype, p, wo, wi, compat), min_frac=1.0)
    g = gpu_bsdf_sample(btype, p, wo, u2)
    c = oracle.bsdf_sample(btype, p, wo, u2)
    c64 = oracle.bsdf_sample(btype, p, wo, u2, fp64=True)
    check_sampling(f"{name}[64k]", btype, g, c, c64)


def test_ggx_fresnel_warps_frames(native, golden):
    n = len(golden["ggx_alpha"])
    D, G1, G, pa = (np.zeros(n, np.float32) for _ in range(4))
    N.call("cl_unit_ggx_eval", P(golden["ggx_alpha"]), P(golden["ggx_m"]), P(golden["ggx_wi"]), P(golden["ggx_wo"]),
           P(D), P(G1), P(G), P(pa), n)
    for a, k in ((D, "ggx_D"), (G1, "ggx_G1"), (G, "ggx_G"), (pa, "ggx_pdfAll")):
        check_ulp(k, a, golden[k], min_frac=1.0)
    m = np.zeros((n, 3), np.float32); pdf = np.zeros(n, np.float32)
    N.call("cl_unit_ggx_sample", P(golden["ggx_alpha"]), P(golden["ggx_u2"]), P(m), P(pdf), n)
    check_vec("ggx.sample.m", m, golden["ggx_sm"], min_frac=0.999)
    check_ulp("ggx.sample.pdf", pdf, golden["ggx_spdf"], min_frac=1.0)
    fc = np.zeros((n, 3), np.float32)
    N.call("cl_unit_fresnel_conductor", P(golden["fres_cos"]), P(golden["fres_eta3"]), P(golden["fres_k3"]), P(fc), n)
    check_ulp("fresnel.conductor", fc, golden["fres_cond"], min_frac=1.0)
    F = np.zeros(n, np.float32); ct = np.zeros(n, np.float32)
    N.call("cl_unit_fresnel_dielectric", P(golden["fres_cos"]), P(golden["fres_eta"]), P(F), P(ct), n)
    check_ulp("fresnel.dielectric.F", F, golden["fres_diel"], min_frac=1.0)
    check_ulp("fresnel.dielectric.cosT", ct, golden["fres_cost"], min_frac=1.0)
    d = np.zeros((n, 2), np.float32); h = np.zeros((n, 3), np.float32)
    N.call("cl_unit_warp", P(golden["warp_u2"]), P(d), P(h), n)
    check_vec("warp.disk", d, golden["warp_disk"], min_frac=0.999)
    # z = sqrt(1 - x^2 - y^2) amplifies the error of x, y by r / z near the rim
    r2 = np.sum(golden["warp_disk"].astype(np.float64) ** 2, axis=1)
    z = np.sqrt(np.maximum(1.0 - r2, 1e-12))
    check_vec("warp.hemisphere", h, golden["warp_hemi"], min_frac=0.98, cond_ulp=4 + 4 * np.sqrt(r2) / z,
              ill=r2 > 1 - 1e-6)
    b = np.zeros((n, 3), np.float32); c = np.zeros((n, 3), np.float32)
    N.call("cl_unit_make_frame", P(golden["mf_a"]), P(b), P(c), n)
    assert ulp_diff(b, golden["mf_b"]).max() == 0 and ulp_diff(c, golden["mf_c"]).max() == 0
    loc = np.zeros((n, 3), np.float32); wld = np.zeros((n, 3), np.float32)
    N.call("cl_unit_frame", P(golden["fr_s"]), P(golden["fr_t"]), P(golden["fr_n"]), P(golden["fr_v"]), P(loc), P(wld), n)
    assert ulp_diff(loc, golden["fr_local"]).max() == 0 and ulp_diff(wld, golden["fr_world"]).max() == 0


def test_directional_and_dome_vs_oracle(native, oracle):
    rng = np.random.default_rng(9)
    n = 1 << 14
    u2 = rng.uniform(0, 1, (n, 2)).astype(np.float32)
    from colvillea_b200 import scenes
    e = scenes.directional()
    p7 = np.array([*e.intensity, *e.direction, e.angular_radius], np.float32)
    dg = np.zeros((n, 3), np.float32); pg = np.zeros(n, np.float32); vg = np.zeros((n, 3), np.float32)
    N.call("cl_unit_directional_sample", P(p7), P(u2), P(dg), P(pg), P(vg), n)
    dc, pc, vc = oracle.directional_sample(p7, u2)
    check_vec("directional.dir", dg, dc)
    check_ulp("directional.pdf", pg, pc, min_frac=1.0)
    assert np.array_equal(vg, vc)
    # HDRI dome: CDF sampling, pdf and lookup against identical (oracle-built) tables
    w, h = 256, 128
    tex = scenes.hdri(w, h, [(d, 2.0, 50.0) for d in scenes.random_upper_dirs(rng, 3)], rng)
    tabs = oracle.dome_build_tables(tex, w, h)
    dg = np.zeros((n, 3), np.float32); pg = np.zeros(n, np.float32); vg = np.zeros((n, 3), np.float32)
    N.call("cl_unit_dome_sample", P(f32(tex)), w, h, *(P(t) for t in tabs), P(u2), P(dg), P(pg), P(vg), n)
    dc, pc, vc = oracle.dome_sample(tex, w, h, tabs, u2)
    check_vec("dome.sample.dir", dg, dc, min_frac=0.999)
    check_ulp("dome.sample.pdf", pg, pc, min_frac=0.999)
    check_vec("dome.sample.value", vg, vc, min_frac=0.999)
    dirs = rng.normal(size=(n, 3)); dirs = f32(dirs / np.linalg.norm(dirs, axis=1, keepdims=True))
    pg = np.zeros(n, np.float32); vg = np.zeros((n, 3), np.float32)
    N.call("cl_unit_dome_pdf_eval", P(f32(tex)), w, h, P(tabs[0]), P(tabs[2]), P(dirs), P(pg), P(vg), n)
    pc, vc = oracle.dome_pdf_eval(tex, w, h, tabs, dirs)
    # sin(acos(y)) is ill-conditioned at the poles; the texel lookup jumps at
    # cell boundaries of u = atan2(x, z) / 2pi, v = acos(y) / pi
    d64 = dirs.astype(np.float64)
    u = np.arctan2(d64[:, 0], d64[:, 2]) * (-0.5 / np.pi) + 0.5
    v = np.arccos(np.clip(d64[:, 1], -1, 1)) / np.pi
    fu, fv = (u * w) % 1.0, (v * h) % 1.0
    edge = (np.minimum(fu, 1 - fu) < 1e-4) | (np.minimum(fv, 1 - fv) < 1e-4) | (1 - np.abs(d64[:, 1]) < 1e-4)
    check_ulp("dome.pdf", pg, pc, min_frac=0.99, ill=edge, rel_ok=1e-4)
    # the bilinear lookup amplifies an atan2/acos ulp difference by the texel
    # gradient: bound it by the FP64 response to a 4e-7 change of u and v
    base = bilinear64(tex, u, v)
    resp = np.zeros(len(u))
    for du, dv in ((4e-7, 0), (-4e-7, 0), (0, 4e-7), (0, -4e-7)):
        resp = np.maximum(resp, np.max(np.abs(bilinear64(tex, u + du, v + dv) - base), axis=1))
    scale = np.max(np.abs(vc.astype(np.float64)), axis=1)
    unit = np.spacing(np.maximum(scale, 1e-30).astype(np.float32)).astype(np.float64)
    check_vec("dome.eval", vg, vc, min_frac=0.99, ill=edge, cond_ulp=4 + resp / unit)


def test_unit_entry_points_reject_bad_input(native):
    L = N.lib()
    assert L.cl_unit_bsdf_eval(3, None, None, None, None, 4) == N.CL_ERR_INVALID_ARG
    assert L.cl_unit_sampler_sequence(None, 1, 1, None) == N.CL_ERR_INVALID_ARG
    # zero-size batches are valid no-ops
    z = np.zeros(1, np.float32)
    assert L.cl_unit_warp(P(z), P(z), P(z), 0) == N.CL_OK


def test_loaded_kernels_are_sm100a(native):
    """The CUDA runtime runs the library's sm_100a SASS (cudaFuncGetAttributes)."""
    import ctypes
    bv, pv = ctypes.c_int32(0), ctypes.c_int32(0)
    N.call("cl_unit_binary_version", ctypes.byref(bv), ctypes.byref(pv))
    assert bv.value == 100, bv.value
