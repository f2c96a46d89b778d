"""Image-quality measurement: relMSE against an FP64-accumulated reference and
the equal-time comparison of neural (guided and/or radiance-cached) and plain
path tracing (no counterpart in the reference renderer, which has neither
networks nor an error metric).

relMSE = mean over pixels and channels of (I - R)^2 / (R^2 + 1e-2).
Equal time: the neural tracer renders `spp` samples per pixel (its time
includes online training); the plain tracer then renders as many samples as
fit in the same device time.  The reference's own noise adds equally to both
relMSE values.  Both use the corrected estimator and the alias
dome sampler; every seed is a disjoint range of progressive frame indices
(the sampler's frame key), and every seed trains a fresh network.
"""
import numpy as np

from . import DOME_ALIAS, FILM_FP64, GuideConfig, RadianceCacheConfig, load_scene

FLAGS = DOME_ALIAS | FILM_FP64
# FLOPs per sample of the guiding MLP (96-64-64-64-64-48, multiply-adds x 2)
INFER_FLOPS = 2 * (96 * 64 + 3 * 64 * 64 + 64 * 48)
# training: forward + input-gradient chain (hash columns only at layer 0) + weight gradients
TRAIN_FLOPS = INFER_FLOPS + 2 * (48 * 64 + 3 * 64 * 64 + 64 * 32) + INFER_FLOPS


def relmse(img, ref):
    img = np.asarray(img, np.float64).reshape(-1, 3)
    ref = np.asarray(ref, np.float64).reshape(-1, 3)
    return float(np.mean((img - ref) ** 2 / (ref * ref + 1e-2)))


def reference(scene, spp, chunk=256, max_depth=None, frame0=1 << 30):
    """FP64-accumulated plain render (mean per pixel, (H*W, 3))."""
    it = load_scene(scene, flags=FLAGS, max_depth=max_depth)
    it.setIterationIndex(frame0)
    done = 0
    while done < spp:
        n = min(chunk, spp - done)
        it.render(n)
        done += n
    s1, _ = it.readbackFilmStats()
    it.close()
    return s1 / spp


def _render(it, spp, frame0):
    it.setIterationIndex(frame0)
    it.render(spp)
    ms = it.stats()["ms_last_render"]
    s1, _ = it.readbackFilmStats()
    return s1 / spp, ms


def equal_time(scene, ref, spp, seeds=3, guide=None, cache=None, max_depth=None, seed_stride=1 << 20):
    """The neural tracer - guiding (`guide`, a GuideConfig) and/or the
    radiance cache (`cache`, a RadianceCacheConfig); guiding alone when both
    are None - renders `spp` samples (training included); the plain tracer
    then renders as many as fit in the same device time.  Over `seeds`
    disjoint frame ranges, every seed with fresh networks.  Returns a dict."""
    if guide is None and cache is None:
        guide = GuideConfig()
    plain = load_scene(scene, flags=FLAGS, max_depth=max_depth)
    _render(plain, 8, 0)                        # warm-up
    ms_probe = _render(plain, 32, 0)[1] / 32    # per-spp cost
    nt = load_scene(scene, flags=FLAGS, max_depth=max_depth)
    out = {"spp_neural": spp, "seeds": seeds, "relmse_neural": [], "relmse_plain": [], "spp_plain": [],
           "ms_neural": [], "ms_plain": [], "train_ms": [], "bias_neural": []}
    for k in range(seeds):
        f0 = (k + 1) * seed_stride
        if guide is not None:
            nt.setGuiding(guide)                # fresh networks, trained online in this render
        if cache is not None:
            nt.setRadianceCache(cache)
        img_n, ms_n = _render(nt, spp, f0)
        tr = (nt.guideStats()["ms_train"] if guide is not None else 0.0) + \
             (nt.cacheStats()["ms_train"] if cache is not None else 0.0)
        n_p = max(1, int(round(ms_n / ms_probe)))
        img_p, ms_p = _render(plain, n_p, f0)
        out["relmse_neural"].append(relmse(img_n, ref))
        out["relmse_plain"].append(relmse(img_p, ref))
        out["bias_neural"].append(float((img_n.mean() - ref.mean()) / ref.mean()))
        out["spp_plain"].append(n_p)
        out["ms_neural"].append(ms_n)
        out["ms_plain"].append(ms_p)
        out["train_ms"].append(tr)
    nt.close()
    plain.close()
    rn, rp = float(np.mean(out["relmse_neural"])), float(np.mean(out["relmse_plain"]))
    out.update({"relmse_neural_mean": rn, "relmse_plain_mean": rp, "plain_over_neural": rp / rn,
                "plain_ms_per_spp": ms_probe})
    return out


def mlp_throughput(scene, guide=None, spp=8, max_depth=None):
    """Inference and training throughput of the guiding network inside a
    guided render (CUDA-event stage timing)."""
    from . import PROFILE_STAGES
    guide = guide if guide is not None else GuideConfig()
    it = load_scene(scene, flags=FLAGS | PROFILE_STAGES, max_depth=max_depth)
    it.setGuiding(guide)
    it.render(guide.train_spp)                  # training phase
    g0 = it.guideStats()
    it.render(spp)
    g1 = it.guideStats()
    it.close()
    n_inf = g1["inferred"] - g0["inferred"]
    ms_inf = g1["ms_infer"]
    steps = max(1, g0["steps"])
    return {"inferred_per_spp": n_inf / spp, "infer_ms_per_spp": ms_inf / spp,
            "infer_tflops": n_inf * INFER_FLOPS / (ms_inf * 1e-3) / 1e12 if ms_inf > 0 else None,
            "train_ms_per_step": g0["ms_train"] / steps,
            "train_samples_per_step": g0["samples_trained"] / steps,
            "train_tflops": g0["samples_trained"] * TRAIN_FLOPS / (g0["ms_train"] * 1e-3) / 1e12
            if g0["ms_train"] > 0 else None,
            "flops_per_sample": {"inference": INFER_FLOPS, "training": TRAIN_FLOPS}}


def equal_spp(scene, ref, spp, variants, seeds=2, max_depth=None, seed_stride=1 << 20):
    """relMSE after `spp` samples per pixel for the plain tracer and for each
    variant (`variants`: name -> GuideConfig, or name -> {"guide": GuideConfig
    or None, "cache": RadianceCacheConfig or None}; a variant's training steps
    are part of its `spp`), over `seeds` disjoint frame ranges with fresh
    networks per seed.  For guiding alone, relMSE at equal spp measures the
    estimators' variance (their bias is zero); with the radiance cache it
    includes the cache's bias (`bias` per variant).  Each entry also gives the
    device time, and `time_ratio` = (plain relMSE x plain time) / (variant
    relMSE x variant time), the equal-time gain of the variant when its error
    falls as 1 / time."""
    plain = load_scene(scene, flags=FLAGS, max_depth=max_depth)
    _render(plain, 8, 0)                         # warm-up
    rows = {}
    r, t = [], []
    for k in range(seeds):
        img, ms = _render(plain, spp, (k + 1) * seed_stride)
        r.append(relmse(img, ref))
        t.append(ms)
    plain.close()
    rows["plain"] = {"relmse": float(np.mean(r)), "ms": float(np.mean(t)), "per_seed": [float(x) for x in r]}
    for name, cfg in variants.items():
        guide, cache = (cfg.get("guide"), cfg.get("cache")) if isinstance(cfg, dict) else (cfg, None)
        it = load_scene(scene, flags=FLAGS, max_depth=max_depth)
        r, t, tr, b = [], [], [], []
        for k in range(seeds):
            if guide is not None:
                it.setGuiding(guide)
            if cache is not None:
                it.setRadianceCache(cache)
            img, ms = _render(it, spp, (k + 1) * seed_stride)
            r.append(relmse(img, ref))
            t.append(ms)
            b.append(float((img.mean() - ref.mean()) / ref.mean()))
            tr.append((it.guideStats()["ms_train"] if guide is not None else 0.0) +
                      (it.cacheStats()["ms_train"] if cache is not None else 0.0))
        it.close()
        rows[name] = {"relmse": float(np.mean(r)), "ms": float(np.mean(t)), "train_ms": float(np.mean(tr)),
                      "per_seed": [float(x) for x in r], "bias": [round(x, 5) for x in b]}
    p = rows["plain"]
    for name, v in rows.items():
        v["spp_ratio"] = p["relmse"] / v["relmse"]
        v["time_ratio"] = (p["relmse"] * p["ms"]) / (v["relmse"] * v["ms"])
    return rows
