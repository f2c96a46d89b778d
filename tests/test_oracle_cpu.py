"""Oracle self-consistency on the CPU: BVH vs brute force, dome tables,
estimator properties (compat vs fixed, Russian roulette, direct lighting)."""
import numpy as np
import pytest

from colvillea_b200 import scenes


@pytest.fixture(scope="module")
def cfg1(oracle):
    s = scenes.config1(0, 64, 64)
    return s, oracle.OracleScene(s.flatten())


def random_rays(rng, n, lo=-6.0, hi=6.0):
    o = rng.uniform(lo, hi, (n, 3))
    o[:, 1] = rng.uniform(0.1, 4.0, n)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3], r[:, 4:7], r[:, 7] = o, d, 3.4e38
    return r


def test_bvh_matches_bruteforce(cfg1):
    _, os_ = cfg1
    rays = random_rays(np.random.default_rng(3), 8000)
    rays[::3, 3] = 0.001
    a, b = os_.trace(rays), os_.trace(rays, bruteforce=True)
    assert np.array_equal(a[1], b[1])
    assert np.array_equal(a[0], b[0])
    assert (a[1] != 0xFFFFFFFF).mean() > 0.2


def test_occluded_consistent_with_closest(cfg1):
    _, os_ = cfg1
    rays = random_rays(np.random.default_rng(4), 4000)
    t, i, _, _ = os_.trace(rays)
    occ = os_.occluded(rays)
    assert np.array_equal(occ.astype(bool), i != 0xFFFFFFFF)


def test_dome_tables_are_cdfs(oracle):
    rng = np.random.default_rng(0)
    tex = scenes.hdri(64, 32, [(d, 4.0, 20.0) for d in scenes.random_upper_dirs(rng, 2)], rng)
    pU, cU, pV, cV = oracle.dome_build_tables(tex, 64, 32)
    cU = cU.reshape(32, 65)
    assert np.all(np.diff(cU, axis=1) >= 0) and np.allclose(cU[:, -1], 1.0, atol=1e-6)
    assert np.all(np.diff(cV) >= 0) and abs(cV[-1] - 1.0) < 1e-6
    # pdf integrates to 1 over the sphere: sum pdf(dir_texel) * dOmega
    d = scenes.texel_directions(64, 32).reshape(-1, 3)
    pdf, _ = oracle.dome_pdf_eval(tex, 64, 32, (pU, cU.ravel(), pV, cV), d)
    th = np.pi * (np.arange(32) + 0.5) / 32
    domega = (2 * np.pi / 64) * (np.pi / 32) * np.sin(th)
    total = (pdf.reshape(32, 64) * domega[:, None]).sum()
    assert abs(total - 1.0) < 2e-3


def test_compat_and_fixed_estimators_differ(cfg1):
    _, os_ = cfg1
    c, _, _ = os_.render(4, max_depth=5, flags=7)
    f, _, _ = os_.render(4, max_depth=5, flags=0)
    assert np.isfinite(c).all() and np.isfinite(f).all()
    assert abs(c.mean() - f.mean()) > 1e-4


def test_russian_roulette_is_unbiased(oracle, cfg1):
    """Fixed estimator with RR from depth 2 vs no RR: equal image means."""
    _, os_ = cfg1
    spp = 64
    a1, a2, _ = os_.render(spp, max_depth=6, rr_start=0, flags=0)
    b1, b2, _ = os_.render(spp, max_depth=6, rr_start=2, flags=0, frame0=5000)
    n = a1.shape[0] * spp
    for c in range(3):
        ma, mb = a1[:, c].sum() / n, b1[:, c].sum() / n
        va = a2[:, c].sum() / n - ma * ma
        vb = b2[:, c].sum() / n - mb * mb
        z = (ma - mb) / np.sqrt(va / n + vb / n)
        assert abs(z) < 4.0, (c, ma, mb, z)


def test_direct_lighting_runs(cfg1, oracle):
    _, os_ = cfg1
    s1, s2, cnt = os_.render(4, flags=oracle.COMPAT_ALL | oracle.DIRECT_LIGHTING)
    assert np.isfinite(s1).all() and cnt[1] > 0
    p1, _, _ = os_.render(4, max_depth=1, flags=oracle.COMPAT_ALL)
    assert s1.sum() > p1.sum()  # direct light adds to the camera-ray environment term


def test_edge_scene_properties(oracle):
    """The checker on the edge-case scenes the GPU tests use: without emitters the film is black and no shadow
    ray is traced; at depth 1 only camera rays are traced; zero-area triangles change no pixel; a view of the sky
    only traces camera rays and sees the dome."""
    import dataclasses
    base = scenes.config1(0, 24, 16)
    n_cam = 24 * 16 * 2

    def run(s, spp=2):
        o = oracle.OracleScene(s.flatten())
        c1, _, cnt = o.render(spp, max_depth=s.max_depth, rr_start=s.rr_start, flags=oracle.COMPAT_ALL)
        return c1, cnt

    c1, cnt = run(dataclasses.replace(base, emitters=[]))
    assert np.all(c1 == 0.0) and int(cnt[1]) == 0 and int(cnt[0]) == n_cam
    c1, cnt = run(dataclasses.replace(base, max_depth=1))
    assert int(cnt[0]) == n_cam and int(cnt[1]) == 0 and c1.max() > 0.0
    ref, rcnt = run(base)
    rng = np.random.default_rng(3)
    p = rng.uniform(-3.0, 3.0, (50, 3)).astype(np.float32)
    pos = np.concatenate([p, p + 1.0, p + 2.0]).astype(np.float32)         # collinear corners
    idx = np.stack([np.arange(50), np.arange(50) + 50, np.arange(50) + 100], 1).astype(np.uint32)
    nv = len(pos)
    mesh = scenes.Mesh(pos, np.tile(np.float32([0, 1, 0]), (nv, 1)), np.tile(np.float32([1, 0, 0]), (nv, 1)),
                       np.zeros((nv, 2), np.float32), idx)
    deg = dataclasses.replace(base, meshes=base.meshes + [mesh],
                              instances=base.instances + [(len(base.meshes), 0, scenes.IDENTITY)])
    c1, cnt = run(deg)
    assert np.array_equal(c1, ref) and np.array_equal(cnt, rcnt)
    sky = dataclasses.replace(base, camera=scenes.look_at_camera((0.0, 3.0, 0.0), (0.0, 100.0, 0.5),
                                                                 (0.0, 0.0, 1.0), 45.0, 24, 16))
    c1, cnt = run(sky)
    assert int(cnt[0]) == n_cam and int(cnt[1]) == 0 and c1.min() > 0.0
