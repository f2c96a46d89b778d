"""Full images of the GPU wavefront integrators against the CPU oracle.

* Same seeds (pcg4d keyed by pixel, frame, counter), reference estimator:
  per-sample arithmetic matches the oracle up to transcendental ulps and the
  FP64-built dome tables, so per-pixel means agree closely.
* Independent seeds: per-pixel Welch tests at 99% on FP64 (sum, sum^2) films;
  the failing fraction must stay within 1% + 3 binomial sigma.
"""
import numpy as np
import pytest
from scipy import stats as sst

import colvillea_b200 as cb
from colvillea_b200 import scenes

pytestmark = pytest.mark.gpu


def welch_fail_fraction(a1, a2, na, b1, b2, nb, alpha=0.01):
    ma, mb = a1 / na, b1 / nb
    va = np.maximum(a2 / na - ma * ma, 0.0) * na / (na - 1)
    vb = np.maximum(b2 / nb - mb * mb, 0.0) * nb / (nb - 1)
    se2 = va / na + vb / nb
    with np.errstate(divide="ignore", invalid="ignore"):
        t = (ma - mb) / np.sqrt(se2)
        df = se2 ** 2 / ((va / na) ** 2 / (na - 1) + (vb / nb) ** 2 / (nb - 1))
    crit = sst.t.ppf(1 - alpha / 2, np.where(np.isfinite(df) & (df > 1), df, 1e9))
    zero = se2 == 0
    fail = np.where(zero, np.abs(ma - mb) > 1e-6 * (np.abs(ma) + 1e-3), np.abs(t) > crit)
    return float(np.mean(fail))


def allowed(nvals, p=0.01):
    return p + 3 * np.sqrt(p * (1 - p) / nvals)


def render_gpu(scene, spp, flags, itype=cb.IntegratorType.WavefrontPathTracing, path_slots=0, **kw):
    it = cb.load_scene(scene, itype=itype, flags=flags | cb.FILM_FP64, path_slots=path_slots, **kw)
    it.render(spp)
    s1, s2 = it.readbackFilmStats()
    img = it.readbackFramebuffer()
    st = it.stats()
    it.close()
    return s1, s2, img, st


@pytest.fixture(scope="module")
def cfg1():
    return scenes.config1(0)


def test_same_seed_reference_estimator(cfg1, oracle):
    s = cfg1
    g1, g2, img, st = render_gpu(s, s.spp, cb.COMPAT_ALL)
    o = oracle.OracleScene(s.flatten())
    c1, c2, cnt = o.render(s.spp, max_depth=s.max_depth, rr_start=s.rr_start, flags=oracle.COMPAT_ALL)
    gm, cm = g1 / s.spp, c1 / s.spp
    rel = np.abs(gm - cm) / (np.abs(cm) + 1e-2)
    print(f"[image] same-seed cfg1: median rel {np.median(rel):.2e}, p99 {np.quantile(rel, 0.99):.2e}, "
          f"max {rel.max():.2e}; mean gpu {gm.mean():.5f} cpu {cm.mean():.5f}; rays gpu "
          f"{st['rays_closest']}/{st['rays_shadow']} cpu {cnt[0]}/{cnt[1]}")
    assert np.quantile(rel, 0.5) < 1e-4
    assert np.quantile(rel, 0.99) < 5e-2
    assert abs(gm.mean() - cm.mean()) / cm.mean() < 2e-3
    # the per-sample paths are the same: identical ray counts up to rare divergences
    assert abs(int(st["rays_closest"]) - int(cnt[0])) < 1e-3 * cnt[0]
    frac = welch_fail_fraction(g1, g2, s.spp, c1, c2, s.spp)
    assert frac <= allowed(g1.size), frac
    # the FP32 film and the FP64 film agree
    assert np.allclose(img[..., :3].reshape(-1, 3), gm, rtol=1e-4, atol=1e-5)


def test_independent_seeds_fixed_estimator_alias(oracle):
    s = scenes.config1(0, 96, 96)
    spp = 64
    flags = cb.DOME_ALIAS
    it = cb.load_scene(s, flags=flags | cb.FILM_FP64)
    it.render(spp)
    g1, g2 = it.readbackFilmStats()
    it.close()
    o = oracle.OracleScene(s.flatten())
    c1, c2, _ = o.render(spp, max_depth=s.max_depth, rr_start=s.rr_start, flags=0, frame0=100000)
    assert np.isfinite(g1).all() and np.isfinite(c1).all()
    frac = welch_fail_fraction(g1, g2, spp, c1, c2, spp)
    print(f"[image] independent cfg1 96x96x{spp}, fixed+alias: Welch fail fraction {frac:.4f} "
          f"(allowed {allowed(g1.size):.4f}); means {g1.mean() / spp:.5f} vs {c1.mean() / spp:.5f}")
    assert frac <= allowed(g1.size)
    tot_g, tot_c = g1.sum(0) / (spp * len(g1)), c1.sum(0) / (spp * len(c1))
    assert np.all(np.abs(tot_g - tot_c) / tot_c < 0.02)


def test_direct_lighting_same_seed(oracle):
    s = scenes.config1(0, 128, 128)
    g1, g2, _, st = render_gpu(s, 8, cb.COMPAT_ALL, itype=cb.IntegratorType.WavefrontDirectLighting)
    o = oracle.OracleScene(s.flatten())
    c1, c2, cnt = o.render(8, max_depth=1, flags=oracle.COMPAT_ALL | oracle.DIRECT_LIGHTING)
    rel = np.abs(g1 - c1) / (np.abs(c1) + 8e-2)
    print(f"[image] DL same-seed: median rel {np.median(rel):.2e}, p99 {np.quantile(rel, 0.99):.2e}")
    assert np.quantile(rel, 0.5) < 1e-4 and np.quantile(rel, 0.99) < 5e-2
    assert welch_fail_fraction(g1, g2, 8, c1, c2, 8) <= allowed(g1.size)


def test_path_regeneration_and_progressive_accumulation():
    """Few path slots (heavy regeneration) and split renders give the same film."""
    s = scenes.config1(0, 64, 64)
    a1, _, _, _ = render_gpu(s, 8, cb.COMPAT_ALL)
    b1, _, _, st = render_gpu(s, 8, cb.COMPAT_ALL, path_slots=777)
    assert np.allclose(a1, b1, rtol=1e-9, atol=1e-9)
    assert st["waves"] > 20
    it = cb.load_scene(s, flags=cb.COMPAT_ALL | cb.FILM_FP64)
    it.render(3)
    it.render(5)
    c1, _ = it.readbackFilmStats()
    assert it.stats()["spp"] == 8 and it.stats()["iteration"] == 8
    assert np.allclose(a1, c1, rtol=1e-9, atol=1e-9)
    # a camera change restarts accumulation (path.h:73-80)
    cam = s.camera.copy()
    cam[0] += 0.5
    it.updateCamera(cam)
    assert it.stats()["spp"] == 0 and it.stats()["iteration"] == 0
    it.updateCamera(cam)  # unchanged camera: no reset
    it.render(1)
    assert it.stats()["spp"] == 1
    it.close()


def test_resize_and_errors(native):
    s = scenes.config1(0, 32, 32)
    it = cb.load_scene(s)
    it.render(1)
    it.resize(48, 40)
    assert it.getFilmSize() == (48, 40)
    it.render(1)
    img = it.readbackFramebuffer()
    assert img.shape == (40, 48, 4) and np.isfinite(img).all()
    with pytest.raises(cb.ClError):
        it.buildMaterials([])
    with pytest.raises(cb.ClError):
        it.buildTLAS([(99, 0, scenes.IDENTITY)])
    with pytest.raises(cb.ClError):
        it.readbackFilmStats()  # FP64 film not enabled
    it.close()
    bad = cb.Integrator.createIntegrator(cb.IntegratorType.WavefrontPathTracing, 8, 8)
    with pytest.raises(cb.ClError):
        bad.render(1)  # nothing built yet
    bad.close()
    # Path slots beyond 2^28 - 1: the traversal kernels' idle-lane mark needs ray indices below that.
    big = cb.load_scene(s, path_slots=1 << 28)
    with pytest.raises(cb.ClError) as e:
        big.render(1)
    assert "path_slots" in str(e.value)
    big.close()


def test_async_readback_pipeline():
    """cl_readback_film_async: each frame's mean arrives intact while the next
    render runs; equal to the synchronous readback and to sum / spp."""
    import torch
    s = scenes.config1(0, 64, 48)
    it = cb.load_scene(s, flags=cb.COMPAT_ALL | cb.FILM_FP64)
    bufs = [torch.empty((48, 64, 4), dtype=torch.float32, pin_memory=True).numpy() for _ in range(3)]
    want = []
    for k in range(3):
        it.render(1)
        want.append(it.readbackFramebuffer().copy())
        it.readbackFramebufferAsync(bufs[k])
        if k < 2:
            it.readbackWait()          # the next readback reuses the staging buffer anyway
    it.render(2)                       # overlaps the last copy
    it.readbackWait()
    for k in range(3):
        np.testing.assert_array_equal(bufs[k], want[k])
    s1, _ = it.readbackFilmStats()
    img = it.readbackFramebuffer()
    np.testing.assert_allclose(img[..., :3].reshape(-1, 3), s1 / 5, rtol=1e-5, atol=1e-6)
    assert np.all(img[..., 3] == 1)
    it.close()
