"""Measures the GPU texture unit as the material textures use it and writes
tests/golden/texture_unit.npz (run on a machine with a B200):

    python tests/golden/gen_texture_unit.py [--out PATH]

The reference reads material textures through CUDA texture objects
(src/core/nodes/textures/imagetex2d.cpp:44-64); so does colvillea_b200
(cl_unit_texture_lookup uses the integrator's texture setup).  The fixture
holds, for seeded inputs:
  w_u, w_out      2x1 RGBA32F texture {0, 1}: u in [0.25, 0.75] -> blend weight
  srgb_table      RGBA8 sRGB, texel i = (i, i, i, i), sampled at texel centres
  unorm_table     the same without sRGB
  f32_tex, f32_uv, f32_out     random RGBA32F 13x7 texture, random uv (wrap)
  u8_tex, u8_uv, u8_out, srgb_out   random RGBA8 11x5 texture, linear and sRGB
The oracle's texture model is checked against it on the CPU
(tests/test_textures.py).
"""
import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import colvillea_b200 as cb  # noqa: E402
from colvillea_b200 import scenes  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "texture_unit.npz"))
    a = ap.parse_args()
    rng = np.random.default_rng(2024)
    out = {}
    t = np.zeros((1, 2, 4), np.float32)
    t[0, 1, 0] = 1.0
    u = (0.25 + 0.5 * np.arange(8193) / 8192).astype(np.float32)
    uv = np.stack([u, np.full_like(u, 0.5)], 1)
    out["w_u"] = u
    out["w_out"] = cb.texture_lookup(scenes.Texture(t), uv)[:, 0]
    ramp = np.repeat(np.arange(256, dtype=np.uint8)[None, :, None], 4, 2)
    cu = ((np.arange(256) + 0.5) / 256).astype(np.float32)
    cuv = np.stack([cu, np.full_like(cu, 0.5)], 1)
    out["srgb_table"] = cb.texture_lookup(scenes.Texture(ramp, srgb=True), cuv)
    out["unorm_table"] = cb.texture_lookup(scenes.Texture(ramp), cuv)
    ft = rng.normal(0, 2, (7, 13, 4)).astype(np.float32)
    fuv = rng.uniform(-3, 3, (4096, 2)).astype(np.float32)
    out["f32_tex"], out["f32_uv"] = ft, fuv
    out["f32_out"] = cb.texture_lookup(scenes.Texture(ft), fuv)
    bt = rng.integers(0, 256, (5, 11, 4)).astype(np.uint8)
    buv = rng.uniform(-3, 3, (4096, 2)).astype(np.float32)
    out["u8_tex"], out["u8_uv"] = bt, buv
    out["u8_out"] = cb.texture_lookup(scenes.Texture(bt), buv)
    out["srgb_out"] = cb.texture_lookup(scenes.Texture(bt, srgb=True), buv)
    np.savez_compressed(a.out, **out)
    print("wrote", a.out)


if __name__ == "__main__":
    main()
