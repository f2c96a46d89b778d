"""The FP64 guiding-network oracle (oracle/pyguide.py) checked on its own:
gradients against central finite differences (smooth mode, no bf16
rounding), the vMF mixture's normalisation, its sampler against its pdf, and
the bf16 rounding helper.  CPU only."""
import numpy as np
import pytest

import pyguide as G


def _unit(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def _params(rng, log2T, scale=0.3):
    T = 1 << log2T
    return np.concatenate([rng.uniform(-scale, scale, G.L_LEVELS * T * 2)] +
                          [rng.uniform(-1, 1, (o, i)).ravel() * np.sqrt(6 / (o + i)) for o, i in G.LAYERS])


@pytest.fixture
def smooth():
    G.ROUND_BF16 = False
    yield
    G.ROUND_BF16 = True


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -9, 1.0 + 3 * 2 ** -9, -2.5, 1e-30, 3.0e38], np.float32)
    r = G.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                        # midpoint of 1 and 1 + 2^-7: ties to even
    assert r[2] == 1.0                        # below the midpoint
    assert r[3] == 1.0 + 2 ** -7              # above the midpoint
    assert r[4] == -2.5
    u = np.asarray(r, np.float32).view(np.uint32)
    assert np.all((u & 0xFFFF) == 0)


def test_gradients_match_finite_differences(smooth):
    rng = np.random.default_rng(1)
    log2T = 8
    res = G.resolutions(4, 64)
    B = 24
    p = _params(rng, log2T)
    pos = rng.uniform(0, 1, (B, 3))
    nrm, wo, om = _unit(rng, B), _unit(rng, B), _unit(rng, B)
    w = rng.uniform(0.1, 2, B)
    loss, g = G.loss_and_grads(p, log2T, res, pos, nrm, wo, om, w)
    nh = G.L_LEVELS * (1 << log2T) * 2
    touched = np.nonzero(g[:nh])[0]
    idx = np.concatenate([rng.choice(touched, 24, replace=False), rng.choice(np.arange(nh, p.size), 48, replace=False)])
    eps = 1e-5
    scale = np.abs(g).max()
    for i in idx:
        q = p.copy(); q[i] += eps
        lp, _ = G.loss_and_grads(q, log2T, res, pos, nrm, wo, om, w)
        q[i] -= 2 * eps
        lm, _ = G.loss_and_grads(q, log2T, res, pos, nrm, wo, om, w)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 * abs(g[i]) + 1e-8 * scale + 1e-11, (i, fd, g[i])


def test_mixture_loss_gradients_match_finite_differences(smooth):
    """Learned selection probability: -log((1-a) p_bsdf + a p_guide)."""
    rng = np.random.default_rng(5)
    log2T = 8
    res = G.resolutions(4, 64)
    B = 24
    p = _params(rng, log2T)
    pos = rng.uniform(0, 1, (B, 3))
    nrm, wo, om = _unit(rng, B), _unit(rng, B), _unit(rng, B)
    w = rng.uniform(0.1, 2, B)
    pb = rng.uniform(0.01, 2.0, B)
    loss, g = G.loss_and_grads(p, log2T, res, pos, nrm, wo, om, w, pb)
    nh = G.L_LEVELS * (1 << log2T) * 2
    touched = np.nonzero(g[:nh])[0]
    idx = np.concatenate([rng.choice(touched, 16, replace=False), rng.choice(np.arange(nh, p.size), 48, replace=False)])
    scale = np.abs(g).max()
    for i in idx:
        q = p.copy(); q[i] += 1e-5
        lp, _ = G.loss_and_grads(q, log2T, res, pos, nrm, wo, om, w, pb)
        q[i] -= 2e-5
        lm, _ = G.loss_and_grads(q, log2T, res, pos, nrm, wo, om, w, pb)
        fd = (lp - lm) / 2e-5
        assert abs(fd - g[i]) <= 1e-6 * abs(g[i]) + 1e-8 * scale + 1e-11, (i, fd, g[i])


def test_head_gradient_matches_finite_differences():
    rng = np.random.default_rng(2)
    out = rng.normal(size=(16, 48))
    out[:, 3:40:5] = rng.uniform(-4, 6, size=(16, 8))  # log kappa inside the clamp
    om = _unit(rng, 16)
    g = G.head_grad(out, om)
    for c in range(40):
        d = np.zeros_like(out); d[:, c] = 1e-6
        fd = (G.log_pdf(out + d, om)[0] - G.log_pdf(out - d, om)[0]) / 2e-6
        np.testing.assert_allclose(fd, g[:, c], rtol=1e-5, atol=1e-7)
    assert np.all(g[:, 40:] == 0)
    pb = rng.uniform(0.05, 1.5, 16)
    gm = G.mix_grad(out, om, pb)
    for c in list(range(41)):
        d = np.zeros_like(out); d[:, c] = 1e-6
        fd = (G.mix_log_pdf(out + d, om, pb) - G.mix_log_pdf(out - d, om, pb)) / 2e-6
        np.testing.assert_allclose(fd, gm[:, c], rtol=1e-5, atol=1e-7)
    assert np.all(gm[:, 41:] == 0)


def test_mixture_is_normalised():
    rng = np.random.default_rng(3)
    out = rng.normal(size=(4, 48))
    out[:, 3:40:5] = rng.uniform(-5, 5, size=(4, 8))
    # Fibonacci sphere quadrature
    n = 400000
    k = np.arange(n) + 0.5
    z = 1 - 2 * k / n
    ph = np.pi * (1 + 5 ** 0.5) * k
    r = np.sqrt(1 - z * z)
    d = np.stack([r * np.cos(ph), r * np.sin(ph), z], 1)
    for b in range(4):
        p = G.mixture_pdf(np.repeat(out[b:b + 1], n, 0), d)
        assert abs(p.mean() * 4 * np.pi - 1) < 2e-3


def test_sampler_matches_pdf():
    """E_p[1/p(X)] = 4 pi and E_p[g(X)/p(X)] = integral of g for samples of
    the mixture sampler - only true when sampler and pdf agree."""
    rng = np.random.default_rng(4)
    out = rng.normal(size=(1, 48))
    out[:, 3:40:5] = rng.uniform(-2, 4, size=(1, 8))
    n = 400000
    o = np.repeat(out, n, 0)
    d, _ = G.vmf_sample(o, rng.uniform(size=(n, 3)))
    np.testing.assert_allclose(np.linalg.norm(d, axis=1), 1, atol=1e-9)
    p = G.mixture_pdf(o, d)
    est = 1 / p
    assert abs(est.mean() - 4 * np.pi) < 4 * est.std() / np.sqrt(n) + 1e-3
    gv = (d[:, 2] > 0.3).astype(float) / p        # integral = 2 pi (1 - 0.3)
    assert abs(gv.mean() - 2 * np.pi * 0.7) < 4 * gv.std() / np.sqrt(n) + 1e-3


def test_hash_grid_indexing():
    res = np.array([3, 100])
    T = 64
    # dense level: (3+1)^3 = 64 <= T
    ix, iy, iz = np.array([1]), np.array([2]), np.array([3])
    assert G.grid_index(ix, iy, iz, 3, T)[0] == 1 + 2 * 4 + 3 * 16
    h = G.grid_index(ix, iy, iz, 100, T)[0]
    assert h == ((1 ^ ((2 * 2654435761) & 0xFFFFFFFF) ^ ((3 * 805459861) & 0xFFFFFFFF)) & (T - 1))
    # p = 1 interpolates the last cell with weight 1
    table = np.arange(2 * 16 * T, dtype=float).reshape(16, T, 2)
    f, corners = G.hash_encode(np.array([[1.0, 1.0, 1.0]]), table, np.array([3] * 16))
    idx, wt = corners[0]
    assert np.isclose(wt[0, 7], 1.0) and idx[0, 7] == 3 + 3 * 4 + 3 * 16


def test_cache_gradients_match_finite_differences(smooth):
    """Radiance cache (96-64-64-16): relative L2 with the stop-gradient
    denominator; the finite difference holds the denominator at the base
    point too, so it is taken on the loss with a frozen denominator."""
    rng = np.random.default_rng(6)
    log2T = 8
    T = 1 << log2T
    res = G.resolutions(4, 64)
    B = 24
    p = np.concatenate([rng.uniform(-0.3, 0.3, G.L_LEVELS * T * 2)] +
                       [rng.uniform(-1, 1, (o, i)).ravel() * np.sqrt(6 / (o + i)) for o, i in G.CACHE_LAYERS])
    pos = rng.uniform(0, 1, (B, 3))
    nrm, wo = _unit(rng, B), _unit(rng, B)
    y = rng.uniform(0, 2, (B, 3))
    loss, g = G.cache_loss_and_grads(p, log2T, res, pos, nrm, wo, y)
    o0 = G.cache_network(p, log2T, res, pos, nrm, wo)[:, :3]
    den = o0 * o0 + 0.01

    def frozen(q):
        o = G.cache_network(q, log2T, res, pos, nrm, wo)[:, :3]
        return np.sum((o - y) ** 2 / den) / (3 * B)

    assert np.isclose(frozen(p), loss)
    nh = G.L_LEVELS * T * 2
    touched = np.nonzero(g[:nh])[0]
    idx = np.concatenate([rng.choice(touched, 16, replace=False), rng.choice(np.arange(nh, p.size), 40, replace=False)])
    scale = np.abs(g).max()
    for i in idx:
        q = p.copy(); q[i] += 1e-5
        lp = frozen(q)
        q[i] -= 2e-5
        lm = frozen(q)
        fd = (lp - lm) / 2e-5
        assert abs(fd - g[i]) <= 1e-6 * abs(g[i]) + 1e-8 * scale + 1e-11, (i, fd, g[i])


@pytest.mark.parametrize("n_min,n_max", [(16, 1024), (4, 512), (16, 2048), (2, 4096), (16, 1000), (8, 8)])
def test_library_level_resolutions_match_the_oracle(native, n_min, n_max):
    """The library's host-side table of hash-grid resolutions (cl_guide_default_resolutions, no GPU needed)
    equals the oracle's floor(n_min b^l), b = (n_max / n_min)^(1/15); with (16, 1024) the finest level is
    1023 (b^15 rounds just below 64)."""
    import colvillea_b200 as cb
    r = cb.default_resolutions(n_min, n_max).astype(np.int64)
    np.testing.assert_array_equal(r, G.resolutions(n_min, n_max))
    assert np.all(np.diff(r) >= 0) and r[0] == n_min
