"""The oracle's restatement against the reference's own code.

tests/golden/ref_kernels.npz holds outputs of the reference's header-only
kernel library (BSDFs, GGX, Fresnel, warps, frames, pcg4d sampler) compiled
on the host from its sources (oracle/ref, generator tests/golden/gen_golden.py).
The oracle must reproduce every value bit for bit.
"""
import numpy as np
import pytest

from conftest import ulp_diff


def test_pcg4d_and_sampler(oracle, golden):
    assert np.array_equal(oracle.pcg4d(golden["pcg4d_in"]), golden["pcg4d_out"])
    seq = oracle.sampler_sequence(golden["sampler_seeds"], golden["sampler_seq"].shape[1])
    assert ulp_diff(seq, golden["sampler_seq"]).max() == 0


@pytest.mark.parametrize("btype,name", [(0, "diffuse"), (1, "conductor"), (2, "dielectric")])
def test_bsdf(oracle, golden, btype, name):
    g = lambda k: golden[f"{name}_{k}"]
    ev = oracle.bsdf_eval(btype, g("params"), g("wo"), g("wi"))
    pdf = oracle.bsdf_pdf(btype, g("params"), g("wo"), g("wi"), compat=True)
    wi, spdf, sval = oracle.bsdf_sample(btype, g("params"), g("wo"), g("u2"))
    assert ulp_diff(ev, g("eval")).max() == 0
    assert ulp_diff(pdf, g("pdf")).max() == 0
    assert ulp_diff(wi, g("swi")).max() == 0
    assert ulp_diff(spdf, g("spdf")).max() == 0
    assert ulp_diff(sval, g("sval")).max() == 0
    # the vectors exercise the non-zero lobes, not only the early outs
    assert (np.abs(ev).sum(1) > 0).sum() > len(ev) // 5
    assert (np.abs(sval).sum(1) > 0).sum() > len(sval) // 5


def test_ggx_fresnel_warps_frames(oracle, golden):
    D, G1, G, pa = oracle.ggx_eval(golden["ggx_alpha"], golden["ggx_m"], golden["ggx_wi"], golden["ggx_wo"])
    for a, k in ((D, "ggx_D"), (G1, "ggx_G1"), (G, "ggx_G"), (pa, "ggx_pdfAll")):
        assert ulp_diff(a, golden[k]).max() == 0, k
    m, p = oracle.ggx_sample(golden["ggx_alpha"], golden["ggx_u2"])
    assert ulp_diff(m, golden["ggx_sm"]).max() == 0 and ulp_diff(p, golden["ggx_spdf"]).max() == 0
    fc = oracle.fresnel_conductor(golden["fres_cos"], golden["fres_eta3"], golden["fres_k3"])
    assert ulp_diff(fc, golden["fres_cond"]).max() == 0
    F, ct = oracle.fresnel_dielectric(golden["fres_cos"], golden["fres_eta"])
    assert ulp_diff(F, golden["fres_diel"]).max() == 0 and ulp_diff(ct, golden["fres_cost"]).max() == 0
    d, h = oracle.warp(golden["warp_u2"])
    assert ulp_diff(d, golden["warp_disk"]).max() == 0 and ulp_diff(h, golden["warp_hemi"]).max() == 0
    b, c = oracle.make_frame(golden["mf_a"])
    assert ulp_diff(b, golden["mf_b"]).max() == 0 and ulp_diff(c, golden["mf_c"]).max() == 0
    loc, wld = oracle.frame(golden["fr_s"], golden["fr_t"], golden["fr_n"], golden["fr_v"])
    assert ulp_diff(loc, golden["fr_local"]).max() == 0 and ulp_diff(wld, golden["fr_world"]).max() == 0


def test_fixed_pdfs_differ_from_reference_only_where_quirks_apply(oracle, golden):
    """compat=False uses the sampling densities instead of the reference's pdf functions (conductor pdfAll(wo),
    diffuse cos(wo), dielectric extra cos(H)); the sampled pdf then equals pdf(wo, wi)."""
    for btype, name in ((0, "diffuse"), (1, "conductor"), (2, "dielectric")):
        g = lambda k: golden[f"{name}_{k}"]
        wi, spdf, sval = oracle.bsdf_sample(btype, g("params"), g("wo"), g("u2"))
        ok = (np.abs(sval).sum(1) > 0) & (spdf > 0)
        fixed = oracle.bsdf_pdf(btype, g("params")[ok], g("wo")[ok], wi[ok], compat=False)
        rel = np.abs(fixed - spdf[ok]) / np.maximum(spdf[ok], 1e-30)
        assert np.median(rel) < 1e-4, name
        assert np.mean(rel < 1e-3) > 0.97, name
