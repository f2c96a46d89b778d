"""Neural radiance cache on the GPU against the FP64 oracle (oracle/pyguide.py):
forward, gradients of the relative L2 loss, training on a known function,
and path tracing that terminates into the cache after a two-bounce prefix."""
import numpy as np
import pytest

import colvillea_b200 as cb
import pyguide as G
from colvillea_b200 import scenes

pytestmark = pytest.mark.gpu

LOG2T = 14


def unit(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def inputs(rng, n):
    return np.concatenate([rng.uniform(0, 1, (n, 3)), unit(rng, n), unit(rng, n)], 1).astype(np.float32)


def make_cache(batch=8192, **kw):
    net = cb.RadianceCacheConfig(network=dict(log2_table=LOG2T, batch=batch, n_min=4, n_max=512, **kw)).network
    return cb.Cache.create(net)


def random_params(c, rng, hash_scale=0.3):
    p = c.get_params()
    nh = p.size - G.mlp_param_count(G.CACHE_LAYERS)
    p[:nh] = rng.uniform(-hash_scale, hash_scale, nh)
    c.set_params(p)
    return c.get_params().astype(np.float64)


def test_cache_forward_matches_oracle():
    rng = np.random.default_rng(20)
    c = make_cache()
    p = random_params(c, rng, 0.5)
    in9 = inputs(rng, 5000)
    out = c.forward(in9).astype(np.float64)
    x = in9.astype(np.float64)
    ref = G.cache_network(p, LOG2T, c.resolutions(), x[:, 0:3], x[:, 3:6], x[:, 6:9])
    err = np.abs(out - ref)
    scale = np.abs(ref).mean()
    print(f"[cache] forward: mean |ref| {scale:.4f}, mean err {err.mean():.2e}, max {err.max():.2e}")
    assert err.mean() < 2e-3 * scale and err.max() < 0.1 * scale
    c.close()


def test_cache_gradient_matches_oracle():
    rng = np.random.default_rng(21)
    c = make_cache()
    p = random_params(c, rng)
    res = c.resolutions()
    in9 = inputs(rng, 4096)
    y = rng.uniform(0, 2, (4096, 3))
    rec = np.concatenate([in9, y], 1).astype(np.float32)
    loss, grad = c.gradient(rec)
    x = rec.astype(np.float64)
    loss_ref, grad_ref = G.cache_loss_and_grads(p, LOG2T, res, x[:, 0:3], x[:, 3:6], x[:, 6:9], x[:, 9:12])
    G.ROUND_BF16 = False
    try:
        _, grad64 = G.cache_loss_and_grads(p, LOG2T, res, x[:, 0:3], x[:, 3:6], x[:, 6:9], x[:, 9:12])
    finally:
        G.ROUND_BF16 = True
    print(f"[cache] loss gpu {loss:.6f} oracle {loss_ref:.6f}")
    assert abs(loss - loss_ref) < 1e-3 * abs(loss_ref) + 1e-6
    nh = p.size - G.mlp_param_count(G.CACHE_LAYERS)
    blocks = [("hash", slice(0, nh))]
    off = nh
    for l, (o, i) in enumerate(G.CACHE_LAYERS):
        blocks.append((f"W{l}", slice(off, off + o * i)))
        off += o * i
    for name, sl in blocks:
        a, b, c64 = grad[sl].astype(np.float64), grad_ref[sl], grad64[sl]
        rel = np.linalg.norm(a - b) / np.linalg.norm(b)
        rel64 = np.linalg.norm(a - c64) / np.linalg.norm(c64)
        relB = np.linalg.norm(b - c64) / np.linalg.norm(c64)
        print(f"[cache] grad {name}: rel err vs BF16 oracle {rel:.2e}, vs FP64 {rel64:.2e} (BF16 oracle vs FP64 "
              f"{relB:.2e})")
        assert rel < 2e-2, name
        assert rel64 < 1.25 * relB + 5e-3, name
    c.close()


def test_cache_learns_a_function():
    """Targets y = a smooth function of position and direction: the relative
    L2 loss drops by an order of magnitude."""
    rng = np.random.default_rng(22)
    c = make_cache(batch=16384)

    def target(x):
        p, wo = x[:, 0:3], x[:, 6:9]
        r = 1.0 + 0.8 * np.sin(3 * p[:, 0]) * np.cos(2 * p[:, 2])
        g = 0.5 + 0.4 * wo[:, 1]
        b = 0.2 + p[:, 1] ** 2
        return np.stack([r, g, b], 1)

    def batch(n):
        x = inputs(rng, n)
        return np.concatenate([x, target(x.astype(np.float64))], 1).astype(np.float32)

    losses = [c.train_step(batch(16384)) for _ in range(300)]
    held = batch(4096)
    pred = c.forward(held[:, :9])[:, :3].astype(np.float64)
    rel = np.mean(np.abs(pred - held[:, 9:12]) / held[:, 9:12])
    print(f"[cache] training: loss {losses[0]:.4f} -> {np.mean(losses[-20:]):.5f}; held-out mean rel err {rel:.4f}")
    assert np.mean(losses[-20:]) < 0.1 * losses[0]
    assert rel < 0.05
    c.close()


def test_cache_integrator_api_errors():
    s = scenes.config1(0, 32, 32)
    dl = cb.load_scene(s, itype=cb.IntegratorType.WavefrontDirectLighting, flags=cb.DOME_ALIAS)
    with pytest.raises(cb.ClError):
        dl.setRadianceCache(cb.RadianceCacheConfig(network=dict(log2_table=12)))
    dl.close()
    comp = cb.load_scene(s, flags=cb.COMPAT_ALL)
    with pytest.raises(cb.ClError):
        comp.setRadianceCache(cb.RadianceCacheConfig(network=dict(log2_table=12)))
    assert comp.cache() is None
    comp.close()


def test_cache_render():
    """Paths end in the cache after two bounces; 1/16 train it.  The image is
    biased but close to the plain tracer's; paths are shorter."""
    s = scenes.config1(0, 128, 128)
    s.max_depth = 8
    spp = 64
    ref = cb.load_scene(s, flags=cb.DOME_ALIAS | cb.FILM_FP64)
    ref.render(1024)
    r1, _ = ref.readbackFilmStats()
    rst = ref.stats()
    ref.close()
    it = cb.load_scene(s, flags=cb.DOME_ALIAS | cb.FILM_FP64)
    it.setRadianceCache(cb.RadianceCacheConfig(network=dict(log2_table=16, batch=1 << 15)))
    it.render(spp)
    g1, _ = it.readbackFilmStats()
    st, cs = it.stats(), it.cacheStats()
    it.close()
    R, I = r1 / 1024, g1 / spp
    bias = (I.mean() - R.mean()) / R.mean()
    rays_plain = rst["rays_closest"] / 1024
    rays_cache = st["last_rays_closest"] / spp
    print(f"[cache] render: relative bias of the image mean {bias:+.4f}; closest rays per spp plain {rays_plain:.0f} "
          f"cache {rays_cache:.0f}; stats {cs}")
    assert np.all(np.isfinite(I))
    assert cs["steps"] == 32 and cs["records_last"] > 1000 and cs["inferred"] > 0 and np.isfinite(cs["last_loss"])
    assert abs(bias) < 0.1
    assert rays_cache < rays_plain   # (this scene's paths are short: most end by escaping before depth 3)
