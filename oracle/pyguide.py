"""ORACLE — test infrastructure only.

FP64 numpy reference of the neural path-guiding network (no counterpart in
the reference renderer; defined by this project): the GPU kernels in
colvillea_b200/csrc/cl_guide.cu are checked against it.

Network:
  * inputs: position p in [0,1]^3 (scene box), shading normal n, outgoing
    direction wo (world space);
  * multiresolution hash grid (Mueller et al. 2022): L = 16 levels, F = 2
    features per level, table of 2^log2T entries per level, resolutions
    floor(nmin * b^l) with b = exp((ln nmax - ln nmin) / (L - 1)); trilinear
    interpolation; dense indexing while (res + 1)^3 <= T, else the spatial
    hash (x * 1) ^ (y * 2654435761) ^ (z * 805459861) mod T;
  * one-blob encoding (Mueller et al. 2019): theta / pi and phi / 2pi + 1/2 of n
    and wo, 16 Gaussian bins each (sigma = 1/16): 64 inputs;
  * MLP 96 -> 64 -> 64 -> 64 -> 64 -> 48, ReLU, no biases;
  * head: 8 von Mises-Fisher lobes, outputs 5k..5k+4 = (mu_xyz, log kappa,
    weight logit); mu = normalize, kappa = exp(clamp(., -5, 7)), softmax
    weights.
Precision (as on the GPU): every matrix operand (weights, activations,
back-propagated deltas) is rounded to bfloat16, sums in FP32/FP64; encoding,
head and loss in FP32/FP64.

Loss over a batch of samples (omega_s, weight w_s):
  loss = -(1/B) sum_s (w_s / mean w) log p(omega_s)
"""
import numpy as np

L_LEVELS, F_FEAT = 16, 2
N_HASH = L_LEVELS * F_FEAT          # 32
N_BLOB = 16                         # bins per scalar
N_IN = N_HASH + 4 * N_BLOB          # 96
WIDTH = 64
N_OUT = 48
N_LOBES = 8
LAYERS = [(WIDTH, N_IN), (WIDTH, WIDTH), (WIDTH, WIDTH), (WIDTH, WIDTH), (N_OUT, WIDTH)]
PRIMES = (1, 2654435761, 805459861)
KAPPA_MIN, KAPPA_MAX = -5.0, 7.0
ROUND_BF16 = True


def bf16(x):
    """Round to bfloat16 (nearest even), returned as float64.  With
    ROUND_BF16 false the value passes through in FP64 (smooth network for the
    finite-difference checks)."""
    if not ROUND_BF16:
        return np.asarray(x, np.float64)
    a = np.ascontiguousarray(np.asarray(x, np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def resolutions(nmin, nmax):
    """Default level resolutions; the tests pass the library's own table
    (cl_guide_default_resolutions) so that both sides index the same grid."""
    b = np.exp((np.log(nmax) - np.log(nmin)) / (L_LEVELS - 1))
    return np.floor(nmin * b ** np.arange(L_LEVELS)).astype(np.int64)


def mlp_param_count(layers=LAYERS):
    return sum(o * i for o, i in layers)


# Radiance cache: 96 -> 64 -> 64 -> 16 (RGB in outputs 0-2).
CACHE_LAYERS = [(WIDTH, N_IN), (WIDTH, WIDTH), (16, WIDTH)]


def split_params(params, log2T, layers=LAYERS):
    """params: flat [hash (L*T*F) | W0 | ... ] (each W row-major [out][in])."""
    T = 1 << log2T
    h = params[: L_LEVELS * T * F_FEAT].reshape(L_LEVELS, T, F_FEAT)
    ws, o = [], L_LEVELS * T * F_FEAT
    for out, inn in layers:
        ws.append(params[o: o + out * inn].reshape(out, inn))
        o += out * inn
    return h, ws


def grid_index(ix, iy, iz, res, T):
    if (res + 1) ** 3 <= T:
        return ix + iy * (res + 1) + iz * (res + 1) ** 2
    h = (ix.astype(np.uint64) * PRIMES[0]) ^ (iy.astype(np.uint64) * PRIMES[1]) ^ (iz.astype(np.uint64) * PRIMES[2])
    return (h & np.uint64(0xFFFFFFFF)).astype(np.int64) & (T - 1)


def hash_encode(pos, table, res):
    """pos (B,3) in [0,1]; table (L,T,F) (bf16 values).  Returns features
    (B,32) and, per level, the 8 corner indices and weights (for backward).
    The cell index is clamped to res - 1, so that p = 1 interpolates the last
    cell with weight 1."""
    B = len(pos)
    T = table.shape[1]
    feats = np.zeros((B, N_HASH))
    corners = []
    p = np.clip(pos.astype(np.float32), 0.0, 1.0)
    for l in range(L_LEVELS):
        x = p * np.float32(res[l])
        i0 = np.minimum(np.floor(x), np.float32(res[l] - 1)).astype(np.int64)
        w = (x - i0.astype(np.float32)).astype(np.float64)
        idxs, wts = [], []
        for c in range(8):
            cx, cy, cz = c & 1, (c >> 1) & 1, (c >> 2) & 1
            wt = (w[:, 0] if cx else 1 - w[:, 0]) * (w[:, 1] if cy else 1 - w[:, 1]) * (w[:, 2] if cz else 1 - w[:, 2])
            idx = grid_index(i0[:, 0] + cx, i0[:, 1] + cy, i0[:, 2] + cz, int(res[l]), T)
            feats[:, 2 * l: 2 * l + 2] += wt[:, None] * table[l, idx]
            idxs.append(idx)
            wts.append(wt)
        corners.append((np.stack(idxs, 1), np.stack(wts, 1)))
    return feats, corners


def one_blob(s):
    centers = (np.arange(N_BLOB) + 0.5) / N_BLOB
    sig = 1.0 / N_BLOB
    return np.exp(-((s[:, None] - centers[None, :]) ** 2) / (2 * sig * sig))


def dir_scalars(d):
    d = d.astype(np.float64)
    th = np.arccos(np.clip(d[:, 2], -1, 1)) / np.pi
    ph = np.arctan2(d[:, 1], d[:, 0]) / (2 * np.pi) + 0.5
    return th, ph


def encode(pos, nrm, wo, table, res):
    hf, corners = hash_encode(pos, table, res)
    nt, nph = dir_scalars(nrm)
    wt, wph = dir_scalars(wo)
    x = np.concatenate([hf, one_blob(nt), one_blob(nph), one_blob(wt), one_blob(wph)], 1)
    return x, corners


def forward(x, ws):
    """MLP with bf16 operands.  Returns head outputs (B,48) and the list of
    layer inputs (bf16-rounded) for backward."""
    acts = []
    h = bf16(x)
    for k, W in enumerate(ws):
        acts.append(h)
        z = h @ bf16(W).T
        if k < len(ws) - 1:
            h = bf16(np.maximum(z, 0.0))
        else:
            h = z
    return h, acts


def head(out):
    """Lobe parameters from head outputs: mu (B,8,3), kappa (B,8), logw (B,8)."""
    o = out[:, :5 * N_LOBES].reshape(-1, N_LOBES, 5)
    raw = o[..., 0:3]
    nrm = np.sqrt(np.sum(raw * raw, -1, keepdims=True))
    mu = raw / np.maximum(nrm, 1e-6)
    lk = np.clip(o[..., 3], KAPPA_MIN, KAPPA_MAX)
    kappa = np.exp(lk)
    logits = o[..., 4]
    logw = logits - np.max(logits, 1, keepdims=True)
    logw = logw - np.log(np.sum(np.exp(logw), 1, keepdims=True))
    return mu, kappa, logw, raw, nrm, o[..., 3]


def vmf_log_norm(kappa):
    # log(kappa / (2 pi (1 - exp(-2 kappa))))
    return np.log(kappa) - np.log(2 * np.pi) - np.log(-np.expm1(-2 * kappa))


def log_pdf(out, omega):
    mu, kappa, logw, *_ = head(out)
    c = np.sum(mu * omega[:, None, :], -1)
    lp = logw + vmf_log_norm(kappa) + kappa * (c - 1.0)
    m = np.max(lp, 1, keepdims=True)
    return (m[:, 0] + np.log(np.sum(np.exp(lp - m), 1))), lp


def head_grad(out, omega):
    """d log p(omega) / d out, (B,48)."""
    mu, kappa, logw, raw, nrm, lkraw = head(out)
    c = np.sum(mu * omega[:, None, :], -1)
    lp = logw + vmf_log_norm(kappa) + kappa * (c - 1.0)
    m = np.max(lp, 1, keepdims=True)
    r = np.exp(lp - m)
    r = r / np.sum(r, 1, keepdims=True)                          # responsibilities
    w = np.exp(logw)
    g = np.zeros((len(out), N_LOBES, 5))
    g[..., 4] = r - w                                            # softmax logits
    e = np.exp(-2 * kappa)
    dlk = 1.0 / kappa - 2 * e / (1 - e) + (c - 1.0)              # d log p_k / d kappa
    inside = (lkraw > KAPPA_MIN) & (lkraw < KAPPA_MAX)
    g[..., 3] = r * dlk * kappa * inside
    dmu = kappa[..., None] * omega[:, None, :]                   # d log p_k / d mu
    proj = dmu - np.sum(dmu * mu, -1, keepdims=True) * mu
    g[..., 0:3] = r[..., None] * proj / np.maximum(nrm, 1e-6)
    out_g = np.zeros_like(out)
    out_g[:, :5 * N_LOBES] = g.reshape(len(out), -1)
    return out_g


SEL_MIN, SEL_MAX = 0.05, 0.95
SEL_OUT = 5 * N_LOBES                  # head output 40: logit of the guide-selection probability


def selection(out):
    """Learned probability of sampling the guide: SEL_MIN + (SEL_MAX - SEL_MIN) sigmoid(o40)."""
    return SEL_MIN + (SEL_MAX - SEL_MIN) / (1.0 + np.exp(-out[:, SEL_OUT]))


def mix_log_pdf(out, omega, pb):
    """log of the one-sample MIS density (1 - a) p_bsdf + a p_guide."""
    a = selection(out)
    pg = np.exp(log_pdf(out, omega)[0])
    return np.log((1 - a) * pb + a * pg)


def mix_grad(out, omega, pb):
    """d log p_mix / d out: the lobe gradient scaled by a p_g / p_mix, and
    (p_g - p_b) / p_mix da/do40 for the selection logit."""
    a = selection(out)
    pg = np.exp(log_pdf(out, omega)[0])
    pm = (1 - a) * pb + a * pg
    g = head_grad(out, omega) * (a * pg / pm)[:, None]
    sg = 1.0 / (1.0 + np.exp(-out[:, SEL_OUT]))
    g[:, SEL_OUT] = (pg - pb) / pm * (SEL_MAX - SEL_MIN) * sg * (1 - sg)
    return g


def loss_and_grads(params, log2T, res, pos, nrm, wo, omega, weight, pb=None, clamp=0.0):
    """Loss and gradient of the flat parameter vector (same layout).  With pb
    (the BSDF pdf of each sample's direction) the objective is the one-sample
    MIS mixture with the learned selection probability, -log p_mix;
    without it, -log p_guide.  clamp > 0: weights above clamp x their mean
    are clamped to it before normalisation."""
    if clamp > 0:
        weight = np.minimum(weight, clamp * np.mean(weight))
    table, ws = split_params(params, log2T)
    tb = bf16(table)
    x, corners = encode(pos, nrm, wo, tb, res)
    out, acts = forward(x, ws)
    if pb is None:
        lp, _ = log_pdf(out, omega)
        hg = head_grad(out, omega)
    else:
        lp = mix_log_pdf(out, omega, pb)
        hg = mix_grad(out, omega, pb)
    wn = weight / np.mean(weight)
    B = len(pos)
    loss = -np.sum(wn * lp) / B
    d = -(wn / B)[:, None] * hg                                  # d loss / d out
    return loss, _backprop(d, ws, acts, table, corners)


def cache_loss_and_grads(params, log2T, res, pos, nrm, wo, target):
    """Radiance cache: relative L2 (o - y)^2 / (o^2 + 0.01) averaged over the
    RGB outputs and the batch, the denominator held constant (stop-gradient)."""
    table, ws = split_params(params, log2T, CACHE_LAYERS)
    tb = bf16(table)
    x, corners = encode(pos, nrm, wo, tb, res)
    out, acts = forward(x, ws)
    o = out[:, :3]
    den = o * o + 0.01
    B = len(pos)
    loss = np.sum((o - target) ** 2 / den) / (3 * B)
    d = np.zeros_like(out)
    d[:, :3] = (2.0 / 3.0) * (o - target) / den / B
    return loss, _backprop(d, ws, acts, table, corners)


def cache_network(params, log2T, res, pos, nrm, wo):
    table, ws = split_params(params, log2T, CACHE_LAYERS)
    x, _ = encode(pos, nrm, wo, bf16(table), res)
    out, _ = forward(x, ws)
    return out


def _backprop(d, ws, acts, table, corners):
    """Gradient of the flat parameter vector from d loss / d out."""
    gws = [None] * len(ws)
    for k in range(len(ws) - 1, -1, -1):
        db = bf16(d)
        gws[k] = db.T @ acts[k]
        d = db @ bf16(ws[k])
        if k > 0:
            d = d * (acts[k] > 0)
    # d: gradient w.r.t. the encoded inputs; hash part scatters to the table
    gt = np.zeros_like(table)
    for l in range(L_LEVELS):
        idx, wt = corners[l]
        for c in range(8):
            for f in range(F_FEAT):
                np.add.at(gt[l, :, f], idx[:, c], wt[:, c] * d[:, 2 * l + f])
    return np.concatenate([gt.ravel()] + [g.ravel() for g in gws])


def adam(params, grad, m, v, step, lr=1e-2, b1=0.9, b2=0.99, eps=1e-10):
    """One Adam step (FP64 here, FP32 on the GPU); step counts from 1."""
    m = b1 * m + (1 - b1) * grad
    v = b2 * v + (1 - b2) * grad * grad
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return params - lr * mh / (np.sqrt(vh) + eps), m, v


def mixture_pdf(out, omega):
    lp, _ = log_pdf(out, omega)
    return np.exp(lp)


def network(params, log2T, res, pos, nrm, wo):
    """Head outputs (B,48) of the network for the given inputs."""
    table, ws = split_params(params, log2T)
    x, _ = encode(pos, nrm, wo, bf16(table), res)
    out, _ = forward(x, ws)
    return out


def vmf_sample(out, u):
    """Mixture sample for head outputs `out` and uniforms u (B,3): lobe by
    u0 over the weights' CDF, direction by Jakob's inversion (2012) with
    u1, u2: w = 1 + log(u1 + (1-u1) e^{-2 kappa}) / kappa, phi = 2 pi u2."""
    mu, kappa, logw, *_ = head(out)
    wts = np.exp(logw)
    cdf = np.cumsum(wts, 1)
    k = np.minimum(np.sum(cdf < (u[:, 0:1] * cdf[:, -1:]), 1), N_LOBES - 1)
    r = np.arange(len(out))
    m, kap = mu[r, k], kappa[r, k]
    w = 1.0 + np.log(u[:, 1] + (1 - u[:, 1]) * np.exp(-2 * kap)) / kap
    w = np.clip(w, -1, 1)
    s = np.sqrt(np.maximum(0.0, 1 - w * w))
    ph = 2 * np.pi * u[:, 2]
    t, b = basis(m)
    d = w[:, None] * m + s[:, None] * (np.cos(ph)[:, None] * t + np.sin(ph)[:, None] * b)
    return d, k


def basis(n):
    """Orthonormal (t, b) with n (Duff et al. 2017 branchless ONB)."""
    sign = np.where(n[:, 2] >= 0, 1.0, -1.0)
    a = -1.0 / (sign + n[:, 2])
    bb = n[:, 0] * n[:, 1] * a
    t = np.stack([1 + sign * n[:, 0] ** 2 * a, sign * bb, -sign * n[:, 0]], 1)
    b = np.stack([bb, sign + n[:, 1] ** 2 * a, -n[:, 1]], 1)
    return t, b
