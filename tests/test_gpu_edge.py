"""Edge cases of the scene description against the CPU oracle, same seeds:
one emitter of each kind alone, no emitter at all, ragged and one-pixel
images, and a zero-sample render call.  The reference's LightSampler picks
among whatever emitters the scene holds (emitter.h:168-202) and its dome
terms vanish without a dome (raygeneration.cu:105-136); its film is any
width x height (path.cpp:53-82)."""
import dataclasses

import numpy as np
import pytest

import colvillea_b200 as cb
from colvillea_b200 import scenes

pytestmark = pytest.mark.gpu


def _render_both(s, spp, gpu_flags, orc_flags, oracle):
    it = cb.load_scene(s, flags=gpu_flags | cb.FILM_FP64)
    it.render(spp)
    g1, _ = it.readbackFilmStats()
    st = it.stats()
    it.close()
    o = oracle.OracleScene(s.flatten())
    c1, _, cnt = o.render(spp, max_depth=s.max_depth, rr_start=s.rr_start, flags=orc_flags)
    return g1 / spp, c1 / spp, st, cnt


def _check_same_seed(gm, cm, st, cnt, label):
    rel = np.abs(gm - cm) / (np.abs(cm) + 1e-2)
    print(f"[edge] {label}: median rel {np.median(rel):.2e}, p99 {np.quantile(rel, 0.99):.2e}; mean gpu "
          f"{gm.mean():.5f} cpu {cm.mean():.5f}; rays gpu {st['rays_closest']}/{st['rays_shadow']} "
          f"cpu {cnt[0]}/{cnt[1]}")
    assert np.isfinite(gm).all()
    assert np.quantile(rel, 0.5) < 1e-4
    assert np.quantile(rel, 0.99) < 5e-2
    assert abs(gm.mean() - cm.mean()) <= 2e-3 * abs(cm.mean()) + 1e-7
    assert abs(int(st["rays_closest"]) - int(cnt[0])) <= max(2, 1e-3 * cnt[0])
    assert abs(int(st["rays_shadow"]) - int(cnt[1])) <= max(2, 1e-3 * cnt[1])


@pytest.mark.parametrize("keep", [scenes.EMIT_DIRECTIONAL, scenes.EMIT_DOME])
@pytest.mark.parametrize("compat", [True, False])
def test_single_emitter(oracle, keep, compat):
    base = scenes.config1(0, 80, 60)
    s = dataclasses.replace(base, emitters=[e for e in base.emitters if e.type == keep])
    assert len(s.emitters) == 1
    gflags, oflags = (cb.COMPAT_ALL, oracle.COMPAT_ALL) if compat else (0, 0)
    gm, cm, st, cnt = _render_both(s, 8, gflags, oflags, oracle)
    kind = "directional" if keep == scenes.EMIT_DIRECTIONAL else "dome"
    _check_same_seed(gm, cm, st, cnt, f"{kind} only, {'reference' if compat else 'corrected'} estimator")
    assert gm.max() > 0.0


def test_no_emitter_renders_black(oracle):
    base = scenes.config1(0, 40, 30)
    s = dataclasses.replace(base, emitters=[])
    gm, cm, st, cnt = _render_both(s, 4, cb.COMPAT_ALL, oracle.COMPAT_ALL, oracle)
    assert np.all(gm == 0.0) and np.all(cm == 0.0)
    assert int(st["rays_shadow"]) == 0 and int(cnt[1]) == 0
    assert abs(int(st["rays_closest"]) - int(cnt[0])) <= 2


@pytest.mark.parametrize("size", [(1, 1), (7, 3), (33, 17)])
def test_ragged_images(oracle, size):
    w, h = size
    s = scenes.config1(0, w, h)
    gm, cm, st, cnt = _render_both(s, 16, cb.COMPAT_ALL, oracle.COMPAT_ALL, oracle)
    assert gm.shape == (w * h, 3)
    if w * h < 100:
        # too few pixels for quantiles: per pixel, with the same tolerance as the median elsewhere
        rel = np.abs(gm - cm) / (np.abs(cm) + 1e-2)
        print(f"[edge] {w}x{h}: max rel {rel.max():.2e}; rays gpu {st['rays_closest']} cpu {cnt[0]}")
        assert np.isfinite(gm).all()
        assert np.mean(rel < 1e-4) >= 0.5
        assert abs(int(st["rays_closest"]) - int(cnt[0])) <= 2
    else:
        _check_same_seed(gm, cm, st, cnt, f"{w}x{h}")


def test_zero_spp_render_is_a_no_op():
    s = scenes.config1(0, 32, 24)
    it = cb.load_scene(s, flags=cb.COMPAT_ALL | cb.FILM_FP64)
    it.render(4)
    a1, a2 = it.readbackFilmStats()
    it.render(0)
    b1, b2 = it.readbackFilmStats()
    it.render(4)
    c1, _ = it.readbackFilmStats()
    it.close()
    assert np.array_equal(a1, b1) and np.array_equal(a2, b2)
    # the zero-sample call did not advance the iteration index: a fresh 8-spp render gives the same film
    it = cb.load_scene(s, flags=cb.COMPAT_ALL | cb.FILM_FP64)
    it.render(8)
    d1, _ = it.readbackFilmStats()
    it.close()
    assert np.allclose(c1, d1, rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize("depth,rr", [(1, 3), (2, 1), (12, 1)])
def test_depth_and_roulette_bounds(oracle, depth, rr):
    """Camera rays only (depth 1), roulette from the first vertex, and deep paths."""
    s = dataclasses.replace(scenes.config1(0, 64, 48), max_depth=depth, rr_start=rr)
    gm, cm, st, cnt = _render_both(s, 8, cb.COMPAT_ALL, oracle.COMPAT_ALL, oracle)
    _check_same_seed(gm, cm, st, cnt, f"max depth {depth}, roulette from {rr}")
    if depth == 1:
        assert int(st["rays_closest"]) == 64 * 48 * 8


@pytest.mark.parametrize("keep", [scenes.EMIT_DIRECTIONAL, scenes.EMIT_DOME])
def test_direct_lighting_single_emitter(oracle, keep):
    base = scenes.config1(0, 64, 48)
    s = dataclasses.replace(base, emitters=[e for e in base.emitters if e.type == keep])
    it = cb.load_scene(s, itype=cb.IntegratorType.WavefrontDirectLighting, flags=cb.COMPAT_ALL | cb.FILM_FP64)
    it.render(8)
    g1, _ = it.readbackFilmStats()
    it.close()
    o = oracle.OracleScene(s.flatten())
    c1, _, _ = o.render(8, max_depth=1, flags=oracle.COMPAT_ALL | oracle.DIRECT_LIGHTING)
    rel = np.abs(g1 - c1) / (np.abs(c1) + 8e-2)
    print(f"[edge] DL, {'directional' if keep == scenes.EMIT_DIRECTIONAL else 'dome'} only: median rel "
          f"{np.median(rel):.2e}, p99 {np.quantile(rel, 0.99):.2e}")
    assert np.isfinite(g1).all() and g1.max() > 0.0
    assert np.quantile(rel, 0.5) < 1e-4 and np.quantile(rel, 0.99) < 5e-2


EXTREME = {
    "conductor alpha 1e-4": scenes.Material(scenes.MAT_METAL, reflectance=(1.0, 1.0, 1.0), roughness=0.01,
                                            eta=scenes.GOLD_ETA, k=scenes.GOLD_K),
    "conductor alpha 1": scenes.Material(scenes.MAT_METAL, reflectance=(1.0, 1.0, 1.0), roughness=1.0,
                                         eta=scenes.GOLD_ETA, k=scenes.GOLD_K),
    "glass alpha 1e-4": scenes.Material(scenes.MAT_GLASS, roughness=0.01, interior_ior=1.5),
    "glass ior 2.4": scenes.Material(scenes.MAT_GLASS, roughness=0.3, interior_ior=2.4),
    "glass ior 1.00001": scenes.Material(scenes.MAT_GLASS, roughness=0.3, interior_ior=1.00001),
    "black diffuse": scenes.Material(scenes.MAT_DIFFUSE, reflectance=(0.0, 0.0, 0.0)),
}


@pytest.mark.parametrize("name", list(EXTREME))
@pytest.mark.parametrize("compat", [True, False])
def test_extreme_materials(oracle, name, compat):
    """Every sphere takes one material at the end of its parameter range (roughness 0.01 and 1, IOR near 1 and
    2.4, zero albedo); the ground stays diffuse.  Near-specular lobes (alpha 1e-4) make per-pixel values huge in
    the reference estimator (its pdf functions), and the same seeds still give the same paths."""
    base = scenes.config1(0, 64, 48)
    s = dataclasses.replace(base, materials=[base.materials[0]] + [EXTREME[name]] * (len(base.materials) - 1))
    gflags, oflags = (cb.COMPAT_ALL, oracle.COMPAT_ALL) if compat else (0, 0)
    gm, cm, st, cnt = _render_both(s, 8, gflags, oflags, oracle)
    _check_same_seed(gm, cm, st, cnt, f"{name}, {'reference' if compat else 'corrected'} estimator")


def test_index_matched_glass_is_rejected():
    """A rough dielectric whose interior IOR equals the exterior's 1.0 has no refraction half-vector
    (roughdielectric.h divides by |wo + eta wi| = 0); the material build refuses it instead of rendering NaN."""
    base = scenes.config1(0, 16, 16)
    s = dataclasses.replace(base, materials=[base.materials[0]] + [
        scenes.Material(scenes.MAT_GLASS, roughness=0.3, interior_ior=1.0)] * (len(base.materials) - 1))
    with pytest.raises(cb.ClError) as e:
        cb.load_scene(s, flags=cb.COMPAT_ALL)
    assert "IOR" in str(e.value)


@pytest.mark.parametrize("view", ["sky", "away"])
def test_every_camera_ray_escapes(oracle, view):
    """A view of the sky only: every camera ray escapes (the escaped-ray class alone, no shading vertex), so the
    film is the dome's radiance and no shadow ray is traced."""
    base = scenes.config1(0, 48, 32)
    pos, at = ((0.0, 3.0, 0.0), (0.0, 100.0, 0.5)) if view == "sky" else ((0.0, 3.0, -40.0), (0.0, 30.0, -100.0))
    s = dataclasses.replace(base, camera=scenes.look_at_camera(pos, at, (0.0, 0.0, 1.0) if view == "sky" else
                                                               (0.0, 1.0, 0.0), 45.0, 48, 32))
    gm, cm, st, cnt = _render_both(s, 4, cb.COMPAT_ALL, oracle.COMPAT_ALL, oracle)
    _check_same_seed(gm, cm, st, cnt, "camera looking up" if view == "sky" else "camera looking away from the scene")
    assert int(st["rays_closest"]) == 48 * 32 * 4 and int(st["rays_shadow"]) == 0
    assert gm.min() > 0.0


def test_degenerate_triangles(oracle, native):
    """Zero-area triangles (a repeated vertex, collinear vertices) mixed into the scene: the builder keeps them,
    no ray hits them, and the image equals the scene's without them."""
    base = scenes.config1(0, 64, 48)
    rng = np.random.default_rng(7)
    n = 300
    p0 = rng.uniform(-4.0, 4.0, (n, 3)).astype(np.float32)
    p0[:, 1] = rng.uniform(0.1, 2.0, n)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    pos = np.concatenate([p0, p0 + d, p0 + 2.0 * d]).astype(np.float32)     # collinear: v, v + d, v + 2d
    idx = np.stack([np.arange(n), np.arange(n) + n, np.arange(n) + 2 * n], 1).astype(np.uint32)
    idx[: n // 2, 2] = idx[: n // 2, 0]                                     # half of them: a repeated vertex
    nv = len(pos)
    nrm = np.tile(np.array([0, 1, 0], np.float32), (nv, 1))
    tan = np.tile(np.array([1, 0, 0], np.float32), (nv, 1))
    mesh = scenes.Mesh(pos, nrm, tan, np.zeros((nv, 2), np.float32), idx)
    s = dataclasses.replace(base, meshes=base.meshes + [mesh],
                            instances=base.instances + [(len(base.meshes), 0, scenes.IDENTITY)])
    gm, cm, st, cnt = _render_both(s, 8, cb.COMPAT_ALL, oracle.COMPAT_ALL, oracle)
    _check_same_seed(gm, cm, st, cnt, "300 zero-area triangles added")
    it = cb.load_scene(base, flags=cb.COMPAT_ALL | cb.FILM_FP64)
    it.render(8)
    b1, _ = it.readbackFilmStats()
    it.close()
    assert np.allclose(gm, b1 / 8, rtol=1e-12, atol=0.0)  # FP64 film sums: atomic order only


def _mirrored_instances_scene():
    """Config 1 with every sphere instance under its own affine map about its centre: a rotation, scales
    U[0.6, 1.4] per axis (ellipsoids) and, for every other sphere, a reflection (negative determinant)."""
    base = scenes.config1(0, 64, 48)
    rng = np.random.default_rng(11)
    inst = [base.instances[0]]
    for k, (mesh_id, mat, _) in enumerate(base.instances[1:]):
        c = base.meshes[mesh_id].positions.astype(np.float64).mean(0)
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        w, x, y, z = q
        R = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                      [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                      [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])
        A = R @ np.diag(rng.uniform(0.6, 1.4, 3))
        if k % 2 == 0:
            A = A @ np.diag([-1.0, 1.0, 1.0])
        M = np.concatenate([A, (c - A @ c)[:, None]], 1)
        inst.append((mesh_id, mat, tuple(float(v) for v in M.ravel())))
    return dataclasses.replace(base, instances=inst)


@pytest.mark.parametrize("two_level", [False, True])
def test_mirrored_and_anisotropic_instances(oracle, two_level):
    """Instance transforms with reflections and unequal axis scales, flattened and as a two-level scene
    (normals by the inverse transpose, the geometric normal flipped for a reflecting map)."""
    s = _mirrored_instances_scene()
    flags = cb.COMPAT_ALL | (cb.TWO_LEVEL if two_level else 0)
    gm, cm, st, cnt = _render_both(s, 8, flags, oracle.COMPAT_ALL, oracle)
    _check_same_seed(gm, cm, st, cnt, f"reflected, anisotropic instances, {'two-level' if two_level else 'flattened'}")
