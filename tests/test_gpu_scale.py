"""Parity at the benchmarked scales: config 2 (1920x1080, 4,685,098 triangles,
2048x1024 dome, depth 8) exactly as bench.py renders it, a reduced config 5
(the same generator: terrain plus rotated and scaled instances, depth 16), and
the integrator's fused guide inference against the standalone network.

* Same seeds, reference estimator with the alias dome sampler: the oracle
  takes the GPU's dome tables (CDF and alias; the tables themselves are
  checked in test_gpu_dome.py) and draws the same pcg4d numbers, so paths
  agree sample by sample up to transcendental ulps.
* Independent seeds, corrected estimator: the GPU's alias sampler against the
  oracle's CDF sampler, per-pixel Welch tests at 99% on FP64 films.
* Hit ids: closest-hit primitive ids and t equal the oracle's (same watertight
  test) apart from flagged exact ties in t; any-hit visibility equal.
"""
import os

import numpy as np
import pytest

import colvillea_b200 as cb
import pyguide as G
from colvillea_b200 import scenes

from test_gpu_render import allowed, welch_fail_fraction
from test_gpu_trace import camera_rays, random_rays

pytestmark = pytest.mark.gpu
THREADS = os.cpu_count() or 8
NO_HIT = 0xFFFFFFFF


def reduced_config5(width=480, height=270):
    """Config 5's generator at a reduced size: a 256^2-vertex terrain and 16
    unique meshes x 12 instances (random rotation, scale U[0.5, 2]), the
    full material mix, 4096x2048 dome, depth 16."""
    return scenes.config5(0, width, height, terrain_n=256, unique=16, copies=12)


def surface_rays(os_, rays, rng):
    """Secondary rays (tmin 1e-3) from the oracle's hit points of `rays`."""
    t, i, _, _ = os_.trace(rays, threads=THREADS)
    hit = i != NO_HIT
    p = rays[hit, 0:3] + t[hit, None] * rays[hit, 4:7]
    d = rng.normal(size=(len(p), 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((len(p), 8), np.float32)
    r[:, 0:3], r[:, 3], r[:, 4:7], r[:, 7] = p, 1e-3, d, 3.4e38
    return r


def world_rays(scene, rng, n):
    """Rays from random points above the terrain in random directions."""
    c = scene.camera
    o = rng.uniform(-40.0, 40.0, (n, 3)) + np.array([0.0, 0.0, 10.0])
    o[:, 1] = rng.uniform(0.5, 6.0, n)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3], r[:, 4:7], r[:, 7] = o, d, 3.4e38
    return r


def check_hits(it, os_, rays, label):
    t, i, b1, b2 = it.traceRays(rays)
    to, io, b1o, b2o = os_.trace(rays, threads=THREADS)
    mismatch = np.nonzero(i != io)[0]
    ties = [k for k in mismatch if t[k] == to[k]]
    print(f"[scale] {label}: {len(rays)} rays, hit fraction {np.mean(i != NO_HIT):.3f}, "
          f"id mismatches {len(mismatch)} (exact ties {len(ties)})")
    assert len(mismatch) == len(ties), f"{len(mismatch) - len(ties)} hit-id mismatches"
    assert len(ties) <= max(2, len(rays) // 10000)
    same = i == io
    assert np.array_equal(t[same], to[same])
    assert np.array_equal(b1[same], b1o[same]) and np.array_equal(b2[same], b2o[same])


def check_any_hit(it, os_, rays, rng):
    rays = rays.copy()
    rays[::5, 7] = rng.uniform(0.5, 20.0, len(rays[::5]))  # finite tmax
    assert np.array_equal(it.occludedRays(rays), os_.occluded(rays, threads=THREADS))


def same_seed_image(scene, spp, label, max_pix_frac=0.02, extra_flags=0, max_median=1e-4, max_ray_diff=1e-3):
    """Reference estimator, alias dome sampler, same seeds: GPU vs oracle."""
    flags = cb.COMPAT_ALL | cb.DOME_ALIAS
    it = cb.load_scene(scene, flags=flags | cb.FILM_FP64 | extra_flags)
    W, H = scene.width, scene.height
    dw, dh = scene.emitters[1].texels.shape[1], scene.emitters[1].texels.shape[0]
    tables = it.domeTables(dw, dh)
    alias = it.domeAliasTables(dw, dh)
    it.render(spp)
    g1, g2 = it.readbackFilmStats()
    st = it.stats()
    it.close()
    import pyoracle
    o = pyoracle.OracleScene(scene.flatten())
    o.set_dome_tables(tables, alias)
    c1, c2, cnt = o.render(spp, max_depth=scene.max_depth, rr_start=scene.rr_start,
                           flags=pyoracle.COMPAT_ALL | pyoracle.DOME_ALIAS, threads=THREADS)
    gm, cm = g1 / spp, c1 / spp
    rel = np.abs(gm - cm) / (np.abs(cm) + 1e-2)
    frac = welch_fail_fraction(g1, g2, spp, c1, c2, spp)
    print(f"[scale] {label} same-seed {W}x{H}x{spp}: median rel {np.median(rel):.2e}, p99 "
          f"{np.quantile(rel, 0.99):.2e}, pixels > 1e-2: {np.mean(rel.max(1) > 1e-2):.4f}; mean gpu "
          f"{gm.mean():.5f} cpu {cm.mean():.5f}; rays gpu {st['rays_closest']}/{st['rays_shadow']} cpu "
          f"{cnt[0]}/{cnt[1]}; Welch fail {frac:.4f}")
    assert np.isfinite(g1).all()
    assert np.median(rel) < max_median
    assert np.mean(rel.max(1) > 1e-2) < max_pix_frac
    assert abs(gm.mean() - cm.mean()) / cm.mean() < 2e-3
    assert abs(int(st["rays_closest"]) - int(cnt[0])) < max_ray_diff * cnt[0]
    assert abs(int(st["rays_shadow"]) - int(cnt[1])) < max_ray_diff * cnt[1]
    assert frac <= allowed(g1.size)


# --- config 2 -----------------------------------------------------------------
@pytest.fixture(scope="module")
def cfg2():
    return scenes.config2(0)


@pytest.fixture(scope="module")
def cfg2_pair(native, oracle, cfg2):
    it = cb.load_scene(cfg2)
    o = oracle.OracleScene(cfg2.flatten())
    yield cfg2, it, o
    it.close()


def test_cfg2_hit_ids(cfg2_pair):
    """65,536 config 2 rays: camera, secondary from camera hits, free rays."""
    s, it, o = cfg2_pair
    st = it.stats()
    assert st["triangles"] == 4685098
    rng = np.random.default_rng(11)
    cam = camera_rays(s, rng, 1 << 15)
    rays = np.concatenate([cam, surface_rays(o, cam[:1 << 14], rng), world_rays(s, rng, 1 << 14)])[:1 << 16]
    check_hits(it, o, rays, f"cfg2 (depth {st['bvh_depth']}, {st['bvh_nodes']} nodes)")
    check_any_hit(it, o, rays, rng)


def test_cfg2_same_seed_image(cfg2):
    """The bench.py workload (reference estimator, alias dome sampler), 2 spp
    over the full 1920x1080 image."""
    same_seed_image(cfg2, 2, "cfg2")


def test_cfg2_independent_seeds_welch(cfg2, oracle):
    """Corrected estimator: the GPU (alias sampler, frames 0-15) against the
    oracle (CDF sampler, other seeds) on 65,536 pixels, 16 spp each."""
    spp = 16
    it = cb.load_scene(cfg2, flags=cb.DOME_ALIAS | cb.FILM_FP64)
    it.render(spp)
    g1, g2 = it.readbackFilmStats()
    it.close()
    rng = np.random.default_rng(5)
    pix = np.sort(rng.choice(cfg2.width * cfg2.height, 1 << 16, replace=False)).astype(np.uint32)
    o = oracle.OracleScene(cfg2.flatten())
    c1, c2, _ = o.render(spp, max_depth=cfg2.max_depth, rr_start=cfg2.rr_start, flags=0, frame0=100000,
                         pixels=pix, threads=THREADS)
    g1, g2 = g1[pix], g2[pix]
    frac = welch_fail_fraction(g1, g2, spp, c1, c2, spp)
    tot_g, tot_c = g1.sum(0) / (spp * len(pix)), c1.sum(0) / (spp * len(pix))
    print(f"[scale] cfg2 independent 65,536 px x {spp}: Welch fail {frac:.4f} (allowed "
          f"{allowed(g1.size):.4f}); channel means {tot_g} vs {tot_c}")
    assert np.isfinite(g1).all() and np.isfinite(c1).all()
    assert frac <= allowed(g1.size)
    assert np.all(np.abs(tot_g - tot_c) / tot_c < 0.03)


# --- reduced config 5 ---------------------------------------------------------
@pytest.fixture(scope="module")
def cfg5r():
    return reduced_config5()


def test_cfg5_reduced_hit_ids(native, oracle, cfg5r):
    s = cfg5r
    it = cb.load_scene(s)
    o = oracle.OracleScene(s.flatten())
    ninst = len(s.instances) - 1
    assert ninst == 192
    rng = np.random.default_rng(12)
    cam = camera_rays(s, rng, 1 << 15)
    rays = np.concatenate([cam, surface_rays(o, cam[:1 << 14], rng), world_rays(s, rng, 1 << 14)])[:1 << 16]
    check_hits(it, o, rays, f"cfg5-reduced ({it.stats()['triangles']} triangles, {ninst} instances)")
    check_any_hit(it, o, rays, rng)
    it.close()


def test_cfg5_reduced_same_seed_image(cfg5r):
    """Depth-16 paths through rotated and scaled instances, 4 spp."""
    same_seed_image(cfg5r, 4, "cfg5-reduced")


# --- two-level instancing (CL_TWO_LEVEL) ---------------------------------------
# The oracle traces the flattened world-space triangles (vertices mapped in
# FP64, rounded to FP32); the GPU maps rays into each instance's object space.
# The two see the same triangle through different roundings: a vertex moves
# by up to about DP (absolute, scene units) between them, which moves the hit
# along the ray by DP / |cos| (cos: ray direction against the triangle's
# normal), so grazing hits differ the most.  Near-ties (a ray through a shared
# edge, or two surfaces within that bound) may resolve to the other triangle.
DP, T_REL = 1e-4, 2e-5


def hit_cosines(flat, prim, d):
    idx = flat.idx[prim]
    p0, p1, p2 = flat.pos[idx[:, 0]].astype(np.float64), flat.pos[idx[:, 1]], flat.pos[idx[:, 2]]
    n = np.cross(p1 - p0, p2 - p0)
    n /= np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-30)
    return np.abs(np.sum(n * d, axis=1))


def check_hits_two_level(it, os_, rays, label, flat):
    t, i, b1, b2 = it.traceRays(rays)
    to, io, _, _ = os_.trace(rays, threads=THREADS)
    hit_g, hit_o = i != NO_HIT, io != NO_HIT
    same = i == io
    eq = same & hit_g
    cos = np.ones(len(rays))
    cos[eq] = hit_cosines(flat, io[eq], rays[eq, 4:7].astype(np.float64))
    tol = DP / np.maximum(cos, 1e-6) + T_REL * np.maximum(np.abs(to), 1.0)
    near = np.abs(t - to) <= tol
    bad = ~same & ~(hit_g & hit_o & (np.abs(t - to) <= DP / 1e-3 + T_REL * np.abs(to)))
    dtc = (np.abs(t - to) * cos)[eq]
    print(f"[scale] {label}: {len(rays)} rays, hit fraction {hit_g.mean():.3f}, id differences {int((~same).sum())} "
          f"(near-ties {int((~same & hit_g & hit_o).sum()) - int(bad.sum())}, other {int(bad.sum())}); on equal ids "
          f"max |dt| {np.abs(t - to)[eq].max() if eq.any() else 0:.2e}, max |dt| cos {dtc.max() if eq.any() else 0:.2e}")
    assert int(bad.sum()) == 0
    assert (~same).mean() < 1e-3
    assert near[eq].all()


def test_cfg5_reduced_two_level_hits(native, oracle, cfg5r):
    """Closest hits and visibility of the two-level scene against the
    oracle's flattened scene; global triangle ids are the flattened ones."""
    s = cfg5r
    it = cb.load_scene(s, flags=cb.COMPAT_ALL | cb.TWO_LEVEL)
    o = oracle.OracleScene(s.flatten())
    st = it.stats()
    assert st["triangles"] == sum(len(s.meshes[m].indices) for m, _, _ in s.instances)
    print(f"[scale] two-level build: {st['ms_bvh_build']:.1f} ms ({st['ms_bvh_build_wall']:.1f} ms wall), top tree "
          f"{st['bvh_nodes']} nodes, depth {st['bvh_depth']}")
    rng = np.random.default_rng(13)
    cam = camera_rays(s, rng, 1 << 15)
    rays = np.concatenate([cam, surface_rays(o, cam[:1 << 14], rng), world_rays(s, rng, 1 << 14)])[:1 << 16]
    check_hits_two_level(it, o, rays, "cfg5-reduced two-level", s.flatten())
    occ_g = it.occludedRays(rays)
    occ_o = o.occluded(rays, threads=THREADS)
    assert np.mean(occ_g != occ_o) < 1e-3
    it.close()


def test_cfg5_reduced_two_level_image(cfg5r):
    """Same-seed image of the two-level scene (depth 16) against the oracle."""
    same_seed_image(cfg5r, 4, "cfg5-reduced two-level", extra_flags=cb.TWO_LEVEL, max_pix_frac=0.05,
                    max_ray_diff=3e-3)


def test_two_level_vertex_edit(native, oracle):
    """A vertex edit of an instanced mesh (refit and rebuild of its tree, the
    top tree rebuilt over the new instance boxes): hits equal the oracle's on
    the edited, flattened scene."""
    s = reduced_config5(160, 90)
    it = cb.load_scene(s, flags=cb.COMPAT_ALL | cb.TWO_LEVEL)
    m = 1                                    # a sphere mesh with 12 rotated, scaled instances
    p = s.meshes[m].positions.copy()
    p *= (1.0 + 0.3 * np.sin(3.0 * p[:, 1:2]))
    rng = np.random.default_rng(14)
    for mode in ("refit", "rebuild"):
        it.updateVertices(m, p, bvh=mode)
        s.meshes[m] = scenes.Mesh(p.astype(np.float32), s.meshes[m].normals, s.meshes[m].tangents, s.meshes[m].uvs,
                                  s.meshes[m].indices)
        flat = s.flatten()
        o = oracle.OracleScene(flat)
        rays = np.concatenate([world_rays(s, rng, 1 << 14), camera_rays(s, rng, 1 << 14)])
        check_hits_two_level(it, o, rays, f"two-level edit ({mode})", flat)
    it.close()


# --- fused guide inference ----------------------------------------------------
def test_fused_guide_inference_matches_network():
    """kGuideInfer (encoding of the hit, tensor-core MLP, head, in one kernel)
    against cl_guide_forward on the same inputs plus the FP64 head: the
    probe's in9 are the rows the fused kernel encoded."""
    s = scenes.config1(0, 256, 256)
    it = cb.load_scene(s, flags=cb.DOME_ALIAS)
    cfg = cb.GuideConfig(log2_table=16, batch=1 << 14, train_spp=8, class_mask=7, bsdf_fraction=0.5)
    it.setGuiding(cfg)
    it.render(8)                                # 8 training steps: a trained, non-trivial network
    rows = it.guideProbe(1 << 15)
    assert len(rows) > 10000
    ray = rows[:, 9].view(np.uint32)
    ok = ray != NO_HIT
    assert ok.mean() > 0.9
    in9, lobes = rows[ok, :9], rows[ok, 10:50]
    assert np.all(np.abs(np.linalg.norm(in9[:, 3:6], axis=1) - 1) < 1e-4)
    assert np.all((in9[:, :3] >= 0) & (in9[:, :3] <= 1))
    out = it.guide().forward(in9)
    mu, kappa, logw = G.head(out.astype(np.float64))[:3]
    w = np.exp(logw) * (1.0 - cfg.bsdf_fraction)
    l4 = lobes[:, :32].reshape(-1, 8, 4)
    err_mu = np.max(np.abs(l4[..., :3] - mu))
    err_k = np.max(np.abs(l4[..., 3] - kappa) / kappa)
    err_w = np.max(np.abs(lobes[:, 32:40] - w))
    print(f"[guide] fused inference, {len(in9)} rows: max |mu| err {err_mu:.2e}, kappa rel {err_k:.2e}, "
          f"weight {err_w:.2e}; weight sum {lobes[:, 32:40].sum(1).mean():.6f}")
    assert err_mu < 1e-5 and err_k < 1e-5 and err_w < 1e-6
    assert np.allclose(lobes[:, 32:40].sum(1), 1.0 - cfg.bsdf_fraction, atol=1e-5)
    # the probe leaves the render state alone: the next spp continues the frame count
    assert it.stats()["spp"] == 8
    it.render(1)
    assert it.stats()["spp"] == 9
    it.close()
