"""The oracle's texture-unit model and normal-mapped frame (no GPU).

The texture model is pinned to measurements of the GPU texture unit
(tests/golden/texture_unit.npz, written by gen_texture_unit.py on a B200
through the same texture setup as the reference's ImageTexture2D,
imagetex2d.cpp:44-64): 8-bit coordinate weights, rounded 8-bit texel
weights, wrap addressing and the 16-bit UNORM result of RGBA8 blends are
reproduced (RGBA32F to FP32 rounding, RGBA8 bit for bit) except where the
unit's coordinate precision moves a weight by one step (about 0.1%); sRGB
lookups stay within the measured 0.007."""
import os

import numpy as np
import pytest

from colvillea_b200 import scenes

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "texture_unit.npz")


@pytest.fixture(scope="module")
def unit():
    return np.load(GOLDEN)


def test_weights_exact(unit, oracle):
    t = np.zeros((1, 2, 4), np.float32)
    t[0, 1, 0] = 1.0
    u = unit["w_u"]
    got = oracle.texture_lookup(scenes.Texture(t), np.stack([u, np.full_like(u, 0.5)], 1))[:, 0]
    np.testing.assert_array_equal(got, unit["w_out"])
    # 257 distinct weights k / 256
    assert len(np.unique(unit["w_out"])) == 257


def check_lookup(got, ref, scale, srgb=False):
    """The model against the unit: RGBA32F and RGBA8 agree to FP32 rounding
    (RGBA8 bit for bit) except where the unit's coordinate precision moves a
    weight by one 1/256 step; sRGB within 0.01 (measured up to 0.0074)."""
    err = np.abs(got.astype(np.float64) - ref) / scale
    if srgb:
        assert np.abs(got[:, :3] - ref[:, :3]).max() < 1e-2
        err = err[:, 3:]
    close = np.all(err < 1e-6, axis=1)
    assert close.mean() > 0.995, close.mean()
    assert err.max() < 2 / 256, err.max()
    return close.mean()


def test_rgba32f_matches_unit(unit, oracle):
    got = oracle.texture_lookup(scenes.Texture(unit["f32_tex"]), unit["f32_uv"])
    check_lookup(got, unit["f32_out"], np.abs(unit["f32_tex"]).max())


def test_rgba8_matches_unit(unit, oracle):
    got = oracle.texture_lookup(scenes.Texture(unit["u8_tex"]), unit["u8_uv"])
    check_lookup(got, unit["u8_out"], 1.0)
    assert np.mean(np.all(got == unit["u8_out"], axis=1)) > 0.995
    i = np.arange(256)
    np.testing.assert_allclose(unit["unorm_table"][:, 0], i / 255.0, rtol=2.0 ** -11, atol=0)


def test_srgb_within_bounds(unit, oracle):
    c = np.arange(256) / 255.0
    curve = np.where(c <= 0.04045, c / 12.92, ((c + 0.055) / 1.055) ** 2.4)
    tab = unit["srgb_table"][:, 0].astype(np.float64)
    rel = np.abs(tab[1:] - curve[1:]) / curve[1:]
    assert tab[0] == 0 and tab[255] == 1 and rel.max() < 6e-3
    assert np.all(np.diff(tab) > 0)                         # monotone
    np.testing.assert_allclose(unit["srgb_table"][:, 3], c, rtol=2.0 ** -11)   # alpha stays linear
    got = oracle.texture_lookup(scenes.Texture(unit["u8_tex"], srgb=True), unit["u8_uv"])
    check_lookup(got, unit["srgb_out"], 1.0, srgb=True)


def test_normal_frame_properties(oracle):
    rng = np.random.default_rng(3)
    n = 4096
    nb = rng.normal(size=(n, 3)); nb /= np.linalg.norm(nb, axis=1, keepdims=True)
    a = rng.normal(size=(n, 3))
    du = a - nb * np.sum(a * nb, 1, keepdims=True); du /= np.linalg.norm(du, axis=1, keepdims=True)
    dv = np.cross(nb, du)
    wo = rng.normal(size=(n, 3)); wo /= np.linalg.norm(wo, axis=1, keepdims=True)
    x = np.zeros((n, 16), np.float32)
    x[:, 0:3], x[:, 3:6], x[:, 6:9], x[:, 9:12] = wo, du, dv, nb
    # the flat texel (0.5, 0.5, 1) maps to the unperturbed normal
    x[:, 12:15] = (0.5, 0.5, 1.0)
    f = oracle.normal_frame(x)
    above = np.sum(wo * nb, 1) > 0
    np.testing.assert_allclose(f[above, 2], nb[above], atol=1e-6)
    np.testing.assert_allclose(f[above, 1], du[above], atol=1e-6)
    # FP32 against FP64, random texels, with the pull-up
    x[:, 12:15] = rng.random((n, 3))
    x[:, 15] = 1
    f32 = oracle.normal_frame(x)
    f64 = oracle.normal_frame(x, fp64=True)
    err = np.abs(f32 - f64).max(axis=(1, 2))
    assert np.quantile(err, 0.99) < 1e-5
