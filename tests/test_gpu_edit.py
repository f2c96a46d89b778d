"""Shape edits on the device (cl_update_mesh_vertices): BVH refit against a
full rebuild, conservative boxes, progressive reset, and the render engine's
compile sequence on the real integrator."""
import copy

import numpy as np
import pytest

import colvillea_b200 as cb
from colvillea_b200 import scenes
from colvillea_b200.engine import RenderEngine, Scene

pytestmark = pytest.mark.gpu


def _xf(rng, scale, t):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    R = np.array([[a*a+b*b-c*c-d*d, 2*(b*c-a*d), 2*(b*d+a*c)],
                  [2*(b*c+a*d), a*a-b*b+c*c-d*d, 2*(c*d-a*b)],
                  [2*(b*d-a*c), 2*(c*d+a*b), a*a-b*b-c*c+d*d]])
    return tuple(float(x) for x in np.concatenate([R * scale, np.asarray(t)[:, None]], 1).reshape(-1))


def instanced_scene(width=96, height=64):
    """A ground quad, one sphere mesh in three instances and one torus mesh in
    two, under rotations, scales and translations."""
    rng = np.random.default_rng(11)
    meshes = [scenes.quad_mesh(12.0), scenes.sphere_mesh(3, (0, 0, 0), 0.8), scenes.torus_mesh(40, 30, (0, 0, 0), 0.7, 0.2)]
    mats = [scenes.Material(scenes.MAT_DIFFUSE, reflectance=(0.5, 0.5, 0.5)),
            scenes.Material(scenes.MAT_METAL, reflectance=(1, 1, 1), roughness=0.4, eta=scenes.GOLD_ETA, k=scenes.GOLD_K),
            scenes.Material(scenes.MAT_DIFFUSE, reflectance=(0.2, 0.6, 0.3))]
    inst = [(0, 0, scenes.IDENTITY),
            (1, 1, _xf(rng, 1.0, (-2.0, 1.0, 0.0))), (1, 2, _xf(rng, 0.6, (0.5, 0.8, 1.5))),
            (1, 1, _xf(rng, 1.4, (2.5, 1.5, 0.5))),
            (2, 2, _xf(rng, 1.0, (0.0, 1.2, -1.5))), (2, 1, _xf(rng, 2.0, (-1.0, 2.5, 2.5)))]
    lobes = [(d, 2.0, 50.0) for d in scenes.random_upper_dirs(rng, 3)]
    ems = [scenes.directional(), scenes.Emitter(scenes.EMIT_DOME, texels=scenes.hdri(128, 64, lobes, rng))]
    cam = scenes.look_at_camera((0, 3, -8), (0, 1, 0), (0, 1, 0), 50.0, width, height)
    return scenes.Scene(width, height, meshes, inst, mats, ems, cam, spp=4, max_depth=5, rr_start=3, name="instanced")


def wobble(m, amp, seed):
    """Smooth displacement along the normals plus a shift: a deformation."""
    rng = np.random.default_rng(seed)
    k = rng.normal(size=3) * 3.0
    p = m.positions.astype(np.float64)
    d = amp * np.sin(p @ k)[:, None] * m.normals + np.array([0.05, 0.1, -0.05])
    return (p + d).astype(np.float32)


def edited(scene, mesh_id, positions):
    s = copy.copy(scene)
    s.meshes = list(scene.meshes)
    m = scene.meshes[mesh_id]
    s.meshes[mesh_id] = scenes.Mesh(positions, m.normals, m.tangents, m.uvs, m.indices)
    return s


def rays_for(scene, n, seed):
    rng = np.random.default_rng(seed)
    f = scene.flatten()
    lo, hi = f.pos.min(0), f.pos.max(0)
    o = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    # half of them camera rays
    cam = np.asarray(scene.camera, np.float64)
    m = n // 2
    u, v = rng.random(m), rng.random(m)
    cd = cam[3:6] + u[:, None] * cam[6:9] + v[:, None] * cam[9:12]
    o[:m] = cam[:3]
    d[:m] = cd / np.linalg.norm(cd, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3], r[:, 3], r[:, 4:7], r[:, 7] = o, 1e-4, d, 1e30
    return r


def check_conservative(nodes, tris):
    """Every present slot's dequantised box (float32, as traversal builds it)
    contains the vertices of all triangles below that slot."""
    n = len(nodes)
    exact = np.zeros((n, 6), np.float64)
    v = tris.reshape(-1, 3, 4)[:, :, :3]
    tlo, thi = v.min(1), v.max(1)
    for i in range(n - 1, -1, -1):
        q = nodes[i]
        p = q[0:3].view(np.float32)
        e = ((q[3] >> np.uint32([0, 8, 16])) & 0xff).astype(np.uint32) << 23
        e = e.view(np.float32)
        imask = int(q[3] >> 24)
        cb_, tb = int(q[4]), int(q[5])
        qlo = [q[8 + 2 * a:10 + 2 * a] for a in range(3)]
        qhi = [q[14 + 2 * a:16 + 2 * a] for a in range(3)]
        lo_all, hi_all = np.full(3, np.inf), np.full(3, -np.inf)
        for s in range(8):
            w, sh = s >> 2, 8 * (s & 3)
            ql = np.array([(int(qlo[a][w]) >> sh) & 0xff for a in range(3)])
            qh = np.array([(int(qhi[a][w]) >> sh) & 0xff for a in range(3)])
            if ql[0] > qh[0]:
                continue
            if imask & (1 << s):
                c = cb_ + bin(imask & ((1 << s) - 1)).count("1")
                blo, bhi = exact[c, :3], exact[c, 3:]
            else:
                meta = (int(q[6 + w]) >> sh) & 0xff
                off, cnt = meta & 31, bin(meta >> 5).count("1")
                blo = tlo[tb + off:tb + off + cnt].min(0)
                bhi = thi[tb + off:tb + off + cnt].max(0)
            dlo = p + e * ql.astype(np.float32)
            dhi = p + e * qh.astype(np.float32)
            assert np.all(dlo <= blo) and np.all(dhi >= bhi), (i, s, dlo, blo, dhi, bhi)
            lo_all, hi_all = np.minimum(lo_all, blo), np.maximum(hi_all, bhi)
        exact[i] = np.concatenate([lo_all, hi_all])


def test_refit_unchanged_is_identical():
    sc = instanced_scene()
    with cb.load_scene(sc) as it:
        n0, t0 = it.bvh()
        it.updateVertices(1, sc.meshes[1].positions, bvh="refit")
        n1, t1 = it.bvh()
        st = it.stats()
        assert st["bvh_refits"] == 1 and st["bvh_rebuilds"] == 0
        np.testing.assert_array_equal(n1, n0)
        np.testing.assert_array_equal(t1, t0)
        # the cost is a sum of double atomics: equal up to summation order
        assert st["bvh_sah_build"] > 1.0 and st["bvh_sah"] == pytest.approx(st["bvh_sah_build"], rel=1e-12)
        print(f"[refit] identity: {st['bvh_nodes']} nodes, {st['triangles']} tris, {st['ms_bvh_update']:.3f} ms, "
              f"build {st['ms_bvh_build']:.3f} ms, SAH {st['bvh_sah']:.2f}")


@pytest.mark.parametrize("mesh_id", [1, 2, 0])
def test_refit_matches_rebuild(mesh_id):
    sc = instanced_scene()
    newp = wobble(sc.meshes[mesh_id], 0.08, mesh_id)
    sc2 = edited(sc, mesh_id, newp)
    rays = rays_for(sc2, 1 << 16, 5 + mesh_id)
    with cb.load_scene(sc) as it, cb.load_scene(sc2) as fresh:
        it.updateVertices(mesh_id, newp, bvh="refit")
        nodes, tris = it.bvh()
        check_conservative(nodes, tris)
        t_r, p_r, b1_r, b2_r = it.traceRays(rays)
        t_f, p_f, b1_f, b2_f = fresh.traceRays(rays)
        hit = p_f != 0xffffffff
        assert hit.mean() > 0.3
        np.testing.assert_array_equal(p_r != 0xffffffff, hit)
        np.testing.assert_array_equal(t_r[hit], t_f[hit])
        same = p_r == p_f
        assert same.mean() > 0.9999, same.mean()
        np.testing.assert_array_equal(b1_r[same & hit], b1_f[same & hit])
        # the same integrator, rebuilt instead: identical hits again
        it.updateVertices(mesh_id, newp, bvh="rebuild")
        t_b, p_b, _, _ = it.traceRays(rays)
        np.testing.assert_array_equal(t_b[hit], t_f[hit])
        st = it.stats()
        assert st["bvh_refits"] == 1 and st["bvh_rebuilds"] == 1


def test_render_after_edit_restarts():
    sc = instanced_scene()
    newp = wobble(sc.meshes[1], 0.1, 7)
    sc2 = edited(sc, 1, newp)
    with cb.load_scene(sc) as it, cb.load_scene(sc2) as fresh:
        it.render(3)
        before = it.readbackFramebuffer().copy()
        it.updateVertices(1, newp, bvh="refit")
        st = it.stats()
        assert st["spp"] == 0 and st["iteration"] == 0
        it.render(4)
        fresh.render(4)
        a, b = it.readbackFramebuffer(), fresh.readbackFramebuffer()
        assert it.stats()["spp"] == 4
        # the film accumulates with float atomics: equal up to summation order
        same = np.all(np.isclose(a, b, rtol=1e-5, atol=1e-6), axis=-1)
        assert same.mean() > 0.999, same.mean()
        assert not np.array_equal(a, before)


def test_auto_policy():
    sc = instanced_scene()
    with cb.load_scene(sc) as it:
        # small motion: refit only
        it.updateVertices(2, wobble(sc.meshes[2], 0.02, 1), bvh="auto")
        st = it.stats()
        assert st["bvh_refits"] == 1 and st["bvh_rebuilds"] == 0
        assert st["bvh_sah"] < 1.5 * st["bvh_sah_build"]
        # the ground quad folded up into a tall wall across the scene: the
        # refitted tree's boxes balloon, auto rebuilds
        q = sc.meshes[0].positions.copy()
        q[:, 1] = np.where(q[:, 0] > 0, 40.0, -40.0) + q[:, 2] * 3.0
        it.updateVertices(0, q, bvh="auto")
        st = it.stats()
        print(f"[refit] auto: sah {st['bvh_sah']:.2f} build {st['bvh_sah_build']:.2f} "
              f"rebuilds {st['bvh_rebuilds']} {st['ms_bvh_update']:.3f} ms")
        if st["bvh_rebuilds"] == 1:
            assert st["bvh_sah"] == st["bvh_sah_build"]
        # scrambled sphere: every triangle of the three sphere instances moves
        # to a random place
        rng = np.random.default_rng(3)
        p = sc.meshes[1].positions[rng.permutation(len(sc.meshes[1].positions))] * 4.0
        it.updateVertices(1, p, bvh="auto")
        st = it.stats()
        print(f"[refit] scrambled: sah {st['bvh_sah']:.2f} build {st['bvh_sah_build']:.2f} "
              f"rebuilds {st['bvh_rebuilds']}")
        assert st["bvh_rebuilds"] >= 1 and st["bvh_sah"] == st["bvh_sah_build"]
        nodes, tris = it.bvh()
        check_conservative(nodes, tris)


def test_update_errors():
    sc = instanced_scene()
    with cb.load_scene(sc) as it:
        p = sc.meshes[1].positions
        with pytest.raises(cb.ClError) as e:
            it.updateVertices(1, p[:-3])
        assert e.value.status == 5
        with pytest.raises(cb.ClError) as e:
            it.updateVertices(9, p)
        assert e.value.status == 5
        bad = p.copy()
        bad[3, 1] = np.inf
        with pytest.raises(cb.ClError) as e:
            it.updateVertices(1, bad)
        assert e.value.status == 5 and "finite" in str(e.value)
        # nothing changed
        assert it.stats()["bvh_refits"] == 0


def test_engine_edit_cycle():
    """Edit -> startRendering on the device gives the image of the edited
    scene rendered from scratch; an unedited frame keeps accumulating."""
    desc = instanced_scene()
    s = Scene.fromScene(desc)
    it = cb.Integrator.createIntegrator(cb.IntegratorType.WavefrontPathTracing, desc.width, desc.height,
                                        cb.RenderConfig(desc.max_depth, desc.rr_start))
    with it:
        eng = RenderEngine(it, s, bvh_update="refit")
        eng.startRendering(2)
        eng.startRendering(2)
        assert it.stats()["spp"] == 4
        newp = wobble(desc.meshes[2], 0.1, 9)
        s.meshes[2].updateVertices(newp)
        s.materials[1].set(roughness=0.2)
        eng.startRendering(4)
        st = it.stats()
        assert st["spp"] == 4 and st["bvh_refits"] == 1
        got = it.readbackFramebuffer().copy()
    desc2 = edited(desc, 2, newp)
    desc2.materials = [copy.copy(m) for m in desc.materials]
    desc2.materials[1].roughness = 0.2
    with cb.load_scene(desc2) as fresh:
        fresh.render(4)
        want = fresh.readbackFramebuffer()
    same = np.all(np.isclose(got, want, rtol=1e-5, atol=1e-6), axis=-1)
    assert same.mean() > 0.999, same.mean()
