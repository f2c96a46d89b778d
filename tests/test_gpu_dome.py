"""HDRI dome preprocessing (FP64 on the device) and alias-table sampling.

* The device tables (reference layout) agree with the reference's FP32
  preprocessing restated in the oracle to FP32 accumulation accuracy.
* The alias sampler returns the CDF sampler's pdf (same table values) and its
  samples follow that density (chi-square over coarse cells).
"""
import numpy as np
import pytest
from scipy import stats as sst

import colvillea_b200 as cb
from colvillea_b200 import scenes
from gpu_util import P, f32
from colvillea_b200 import _native as N

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dome_scene():
    s = scenes.config1(0, 16, 16)
    it = cb.load_scene(s, flags=cb.COMPAT_ALL | cb.DOME_ALIAS)
    yield s, it
    it.close()


def test_tables_match_reference_preprocessing(dome_scene, oracle):
    s, it = dome_scene
    tex = s.dome().texels
    h, w = tex.shape[:2]
    g = it.domeTables(w, h)
    c = oracle.dome_build_tables(tex, w, h)
    names = ("pUcondV_c", "CDFpUcondV", "pV_c", "CDFpV")
    for name, a, b in zip(names, g, c):
        rel = np.abs(a.astype(np.float64) - b) / (np.abs(b) + 1e-12)
        print(f"[dome] {name}: max rel {rel.max():.2e}")
        assert rel.max() < 2e-4, name
    cU = g[1].reshape(h, w + 1)
    assert np.all(np.diff(cU, axis=1) >= 0) and np.all(cU[:, -1] == 1.0)
    assert np.all(np.diff(g[3]) >= 0) and g[3][-1] == 1.0


def test_alias_sampler_pdf_and_distribution(dome_scene):
    s, it = dome_scene
    tex = s.dome().texels
    h, w = tex.shape[:2]
    n = 1 << 20
    u2 = np.random.default_rng(5).uniform(0, 1, (n, 2)).astype(np.float32)
    d, pdf, val = it.domeAliasSample(u2)
    assert np.all(pdf > 0) and np.isfinite(d).all()
    # pdf equals the pdf lookup of the sampled direction (same tables) except at cell edges
    pU, cU, pV, cV = it.domeTables(w, h)
    pe = np.zeros(n, np.float32); ve = np.zeros((n, 3), np.float32)
    N.call("cl_unit_dome_pdf_eval", P(f32(tex)), w, h, P(pU), P(pV), P(f32(d)), P(pe), P(ve), n)
    rel = np.abs(pe - pdf) / pdf
    print(f"[alias] pdf == lookup for {np.mean(rel < 1e-5):.5f} of samples")
    assert np.mean(rel < 1e-5) > 0.995
    # distribution: counts over 32x16 coarse cells vs the table density
    d64 = d.astype(np.float64)
    u = np.arctan2(d64[:, 0], d64[:, 2]) * (-0.5 / np.pi) + 0.5
    v = np.arccos(np.clip(d64[:, 1], -1, 1)) / np.pi
    cu, cv = 32, 16
    iu = np.clip((u * cu).astype(int), 0, cu - 1); iv = np.clip((v * cv).astype(int), 0, cv - 1)
    obs = np.bincount(iv * cu + iu, minlength=cu * cv).astype(np.float64)
    f = pU.reshape(h, w + 1)[:, :w].astype(np.float64)
    exp = f.reshape(cv, h // cv, cu, w // cu).sum(axis=(1, 3)).ravel()
    exp = exp / exp.sum() * n
    keep = exp > 20
    chi2 = np.sum((obs[keep] - exp[keep]) ** 2 / exp[keep])
    p = sst.chi2.sf(chi2, keep.sum() - 1)
    print(f"[alias] chi2 {chi2:.1f} over {keep.sum()} cells, p = {p:.3g}")
    assert p > 1e-4


def dome_tables_fp64(tex):
    """The tables of one dome in FP64 (numpy), for the two device paths."""
    h, w = tex.shape[:2]
    t = tex.astype(np.float64)
    lum = t[..., 0] * 0.212671 + t[..., 1] * 0.71516 + t[..., 2] * 0.072169
    wgt = np.sin(np.pi * (np.arange(h) + 0.5) / h)[:, None] * lum
    rows = wgt.sum(axis=1)
    with np.errstate(invalid="ignore", divide="ignore"):
        cdf = np.where(rows[:, None] > 0, np.cumsum(wgt, axis=1) / rows[:, None], np.arange(1, w + 1) / w)
        pdf = np.where(rows[:, None] > 0, wgt / rows[:, None], 1.0 / w)
    rc = rows / w
    return wgt, cdf, pdf, rc, np.cumsum(rc) / rc.sum(), rc / rc.sum()


def alias_row_mass(col, w, h):
    prob = col[0::2].view(np.float32).astype(np.float64).reshape(h, w)
    alias = col[1::2].astype(np.int64).reshape(h, w)
    assert np.all((prob >= 0) & (prob <= 1)) and np.all((alias >= 0) & (alias < w))
    mass = prob.copy()
    np.add.at(mass, (np.broadcast_to(np.arange(h)[:, None], (h, w)), alias), 1.0 - prob)
    return mass / w


@pytest.mark.parametrize("w,h", [(16384, 12), (20480, 6)], ids=["block-per-row", "thread-per-row"])
def test_wide_rows_both_paths(w, h):
    """Rows of 16,384 texels take the shared-memory kernels (one block per
    row), wider ones the thread-per-row kernels; both against FP64 numpy,
    with a black row and a black band of columns."""
    rng = np.random.default_rng(w)
    tex = scenes.hdri(w, h, [(d, 2.0, 300.0) for d in scenes.random_upper_dirs(rng, 4)], rng)
    tex[h // 2] = 0.0
    tex[:, w // 5: w // 5 + 700] = 0.0
    it = cb.Integrator.createIntegrator(cb.IntegratorType.WavefrontPathTracing, 8, 8)
    try:
        it.buildEmitters([scenes.Emitter(scenes.EMIT_DOME, texels=tex)])
        pU, cU, pV, cV = it.domeTables(w, h)
        ar, ac = it.domeAliasTables(w, h)
    finally:
        it.close()
    wgt, cdf, pdf, rc, cdfV, pdfV = dome_tables_fp64(tex)
    pU = pU.reshape(h, w + 1); cU = cU.reshape(h, w + 1)
    np.testing.assert_allclose(pU[:, :w], wgt, rtol=3e-7, atol=0)
    np.testing.assert_allclose(pU[:, w], rc, rtol=3e-7, atol=0)
    np.testing.assert_allclose(cU[:, 1:], cdf, rtol=3e-7, atol=1e-12)
    assert np.all(cU[:, 0] == 0) and np.all(cU[:, w] == 1) and np.all(np.diff(cU, axis=1) >= 0)
    assert np.all(pU[h // 2] == 0)
    np.testing.assert_allclose(pV[:h], rc, rtol=3e-7, atol=0)
    np.testing.assert_allclose(cV[1:], cdfV, rtol=3e-7, atol=1e-12)
    assert cV[0] == 0 and cV[h] == 1 and np.all(np.diff(cV) >= 0)
    np.testing.assert_allclose(alias_row_mass(ac, w, h), pdf, rtol=1e-4, atol=1e-12)
    np.testing.assert_allclose(alias_row_mass(ar, h, 1)[0], pdfV, rtol=1e-4, atol=1e-12)
    black = ac.reshape(h, w, 2)[h // 2]
    assert np.all(black[:, 1] == np.arange(w)) and np.all(black[:, 0].view(np.float32) == 1.0)
