"""A scene loaded from OBJ and Radiance .hdr files renders the same image as
the scene built from arrays: per-triangle geometry identical, per-pixel means
within the 99% Welch test (the loader's tangents come from the uvs, so only the
orientation of the sampling frame differs)."""
import numpy as np
import pytest

import colvillea_b200 as cb
from colvillea_b200 import scenes

from test_gpu_render import allowed, welch_fail_fraction
from test_io import rgbe_decode, rgbe_encode, write_hdr

pytestmark = pytest.mark.gpu


def test_scene_from_files(tmp_path):
    s = scenes.config1(0, 96, 96)
    dome = s.dome()
    q = rgbe_encode(dome.texels[..., :3].astype(np.float64))
    write_hdr(tmp_path / "dome.hdr", q, rle=True)
    dome.texels = rgbe_decode(q)                      # both scenes light with the quantised dome
    scenes.save_obj(tmp_path / "scene.obj", s.meshes)
    meshes = cb.load_obj(tmp_path / "scene.obj")
    assert len(meshes) == len(s.meshes)
    for a, b in zip(s.meshes, meshes):
        for attr in ("positions", "normals", "uvs"):
            np.testing.assert_array_equal(getattr(a, attr)[a.indices], getattr(b, attr)[b.indices])
        np.testing.assert_allclose(np.abs(np.sum(b.normals * b.tangents, 1)), 0, atol=1e-5)
    loaded = scenes.Scene(s.width, s.height, meshes, s.instances, s.materials,
                          [e if e.type != scenes.EMIT_DOME else
                           scenes.Emitter(scenes.EMIT_DOME, texels=cb.load_hdr(tmp_path / "dome.hdr"))
                           for e in s.emitters], s.camera, s.spp, s.max_depth, s.rr_start)
    np.testing.assert_array_equal(loaded.dome().texels, dome.texels)
    spp = 128
    out = []
    for sc in (s, loaded):
        it = cb.load_scene(sc, flags=cb.DOME_ALIAS | cb.FILM_FP64)
        it.render(spp)
        out.append(it.readbackFilmStats())
        it.close()
    (a1, a2), (b1, b2) = out
    frac = welch_fail_fraction(a1, a2, spp, b1, b2, spp)
    print(f"[io] OBJ/HDR scene vs arrays: Welch fail {frac:.4f} (allowed {allowed(a1.size):.4f}); "
          f"means {a1.mean() / spp:.5f} {b1.mean() / spp:.5f}")
    assert frac <= allowed(a1.size)
    assert abs(a1.mean() - b1.mean()) / a1.mean() < 5e-3
    # film output
    img = np.concatenate([b1.reshape(s.height, s.width, 3) / spp, np.ones((s.height, s.width, 1))], -1)
    cb.write_pfm(tmp_path / "film.pfm", img)
    np.testing.assert_array_equal(cb.read_pfm(tmp_path / "film.pfm")[..., :3], img[..., :3].astype(np.float32))
