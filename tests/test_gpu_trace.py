"""The 8-wide BVH traversal against a brute-force intersector: closest-hit
primitive ids and t must match exactly (shared watertight test), apart from
flagged exact ties; any-hit visibility must match."""
import numpy as np
import pytest

import colvillea_b200 as cb
from colvillea_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cfg1_pair(native, oracle):
    s = scenes.config1(0)
    it = cb.load_scene(s)
    return s, it, oracle.OracleScene(s.flatten())


def camera_rays(scene, rng, n):
    c = scene.camera
    pos, d00, ddu, ddv = c[0:3], c[3:6], c[6:9], c[9:12]
    u, v = rng.uniform(0, 1, n), rng.uniform(0, 1, n)
    d = d00[None] + u[:, None] * ddu[None] + v[:, None] * ddv[None]
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3], r[:, 4:7], r[:, 7] = pos, d, 3.4e38
    return r


def random_rays(rng, n):
    o = rng.uniform(-6.0, 6.0, (n, 3))
    o[:, 1] = rng.uniform(0.05, 4.0, n)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3], r[:, 4:7], r[:, 7] = o, d, 3.4e38
    return r


def surface_rays(os_, rays, rng):
    """Secondary rays from the hit points of `rays` (tmin = 1e-3), random directions."""
    t, i, _, _ = os_.trace(rays)
    hit = i != 0xFFFFFFFF
    p = rays[hit, 0:3] + t[hit, None] * rays[hit, 4:7]
    d = rng.normal(size=(len(p), 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((len(p), 8), np.float32)
    r[:, 0:3], r[:, 3], r[:, 4:7], r[:, 7] = p, 1e-3, d, 3.4e38
    return r


def test_closest_hit_matches_bruteforce(cfg1_pair):
    s, it, os_ = cfg1_pair
    rng = np.random.default_rng(1)
    prim = camera_rays(s, rng, 1 << 15)
    rays = np.concatenate([prim, random_rays(rng, 1 << 15), surface_rays(os_, prim[:8192], rng)])
    t, i, b1, b2 = it.traceRays(rays)
    tb, ib, b1b, b2b = os_.trace(rays, bruteforce=True)
    mismatch = np.nonzero(i != ib)[0]
    # a mismatch is only allowed as a flagged exact tie in t
    ties = [k for k in mismatch if t[k] == tb[k]]
    assert len(mismatch) == len(ties), f"{len(mismatch) - len(ties)} hit-id mismatches of {len(rays)}"
    assert len(ties) <= len(rays) // 10000
    same = i == ib
    assert np.array_equal(t[same], tb[same])
    assert np.array_equal(b1[same], b1b[same]) and np.array_equal(b2[same], b2b[same])
    print(f"[trace] {len(rays)} rays, hits {np.mean(i != 0xFFFFFFFF):.3f}, ties {len(ties)}")


def test_any_hit_matches(cfg1_pair):
    s, it, os_ = cfg1_pair
    rng = np.random.default_rng(2)
    rays = np.concatenate([random_rays(rng, 1 << 15), surface_rays(os_, camera_rays(s, rng, 8192), rng)])
    rays[::7, 7] = rng.uniform(0.5, 5.0, len(rays[::7]))  # finite tmax
    occ = it.occludedRays(rays)
    assert np.array_equal(occ, os_.occluded(rays))


def test_edge_cases(cfg1_pair):
    s, it, os_ = cfg1_pair
    # empty batch
    t, i, _, _ = it.traceRays(np.zeros((0, 8), np.float32))
    assert len(t) == 0
    # axis-aligned directions, rays along the ground plane, ray from below the ground
    r = np.zeros((6, 8), np.float32)
    r[:, 7] = 3.4e38
    r[0, 0:3], r[0, 4:7] = (0, 5, 0), (0, -1, 0)
    r[1, 0:3], r[1, 4:7] = (-9, 0, 0.3), (1, 0, 0)
    r[2, 0:3], r[2, 4:7] = (0, -1, 0), (0, 1, 0)
    r[3, 0:3], r[3, 4:7] = (30, 1, 30), (0, 0, 1)
    r[4, 0:3], r[4, 4:7] = (0.5, 3, 0.5), (0, 0, -1)
    r[5, 0:3], r[5, 4:7], r[5, 7] = (0, 5, 0), (0, -1, 0), 1.0  # tmax before the ground
    t, i, _, _ = it.traceRays(r)
    tb, ib, _, _ = os_.trace(r, bruteforce=True)
    assert np.array_equal(i, ib) and np.array_equal(t[i != 0xFFFFFFFF], tb[ib != 0xFFFFFFFF])


def test_bvh_shape_and_stats(cfg1_pair):
    s, it, os_ = cfg1_pair
    st = it.stats()
    assert st["triangles"] == s.num_triangles == 10242
    assert 0 < st["bvh_nodes"] < st["triangles"] and st["bvh_depth"] < 40
    rays = camera_rays(s, np.random.default_rng(5), 4096)
    nodes, tris = it.traceStats(rays)
    assert nodes > 0 and tris > 0
    print(f"[bvh] nodes {st['bvh_nodes']} depth {st['bvh_depth']} build {st['ms_bvh_build']:.2f} ms; "
          f"per camera ray: {nodes / 4096:.1f} nodes, {tris / 4096:.1f} tris")


def test_single_and_few_triangles(native, oracle):
    """Trees with 1, 2 and 5 triangles (root as a leaf slot, tiny inner trees)."""
    rng = np.random.default_rng(3)
    for ntri in (1, 2, 5):
        m = scenes.quad_mesh(4.0)
        pos = rng.uniform(-2, 2, (3 * ntri, 3)).astype(np.float32)
        idx = np.arange(3 * ntri, dtype=np.uint32).reshape(-1, 3)
        nrm = np.tile(np.array([0, 1, 0], np.float32), (3 * ntri, 1))
        mesh = scenes.Mesh(pos, nrm, np.tile(np.array([1, 0, 0], np.float32), (3 * ntri, 1)),
                           np.zeros((3 * ntri, 2), np.float32), idx)
        sc = scenes.Scene(8, 8, [mesh], [(0, 0, scenes.IDENTITY)], [scenes.Material(0, (0.5, 0.5, 0.5))],
                          [scenes.directional()], scenes.look_at_camera((0, 3, -10), (0, 0, 0), (0, 1, 0), 45, 8, 8))
        it = cb.load_scene(sc)
        os_ = oracle.OracleScene(sc.flatten())
        o = rng.uniform(-3, 3, (4096, 3)); tgt = pos[rng.integers(0, len(pos), 4096)] + rng.normal(0, 0.3, (4096, 3))
        d = tgt - o; d /= np.linalg.norm(d, axis=1, keepdims=True)
        r = np.zeros((4096, 8), np.float32); r[:, 0:3], r[:, 4:7], r[:, 7] = o, d, 3.4e38
        t, i, _, _ = it.traceRays(r)
        tb, ib, _, _ = os_.trace(r, bruteforce=True)
        assert np.array_equal(i, ib), ntri
        it.close()
