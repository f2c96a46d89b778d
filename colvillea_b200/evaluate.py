"""Image-quality measurement: relMSE against an FP64-accumulated reference and
the equal-time comparison of guided and plain path tracing (no counterpart in
the reference renderer, which has neither guiding nor an error metric).

relMSE = mean over pixels and channels of (I - R)^2 / (R^2 + 1e-2).
Equal time: the guided tracer renders `spp` samples per pixel (its time
includes online training); the plain tracer then renders as many samples as
fit in the same device time.  Both use the corrected estimator and the alias
dome sampler; every seed is a disjoint range of progressive frame indices
(the sampler's frame key), and every seed trains a fresh network.
"""
import numpy as np

from . import DOME_ALIAS, FILM_FP64, GuideConfig, load_scene

FLAGS = DOME_ALIAS | FILM_FP64
# FLOPs per sample of the guiding MLP (96-64-64-64-64-48, multiply-adds x 2)
INFER_FLOPS = 2 * (96 * 64 + 3 * 64 * 64 + 64 * 48)
# training: forward + input-gradient chain (hash columns only at layer 0) + weight gradients
TRAIN_FLOPS = INFER_FLOPS + 2 * (48 * 64 + 3 * 64 * 64 + 64 * 32) + INFER_FLOPS


def relmse(img, ref):
    img = np.asarray(img, np.float64).reshape(-1, 3)
    ref = np.asarray(ref, np.float64).reshape(-1, 3)
    return float(np.mean((img - ref) ** 2 / (ref * ref + 1e-2)))


def reference(scene, spp, chunk=256, max_depth=None, frame0=0):
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


def equal_time(scene, ref, spp, seeds=3, guide=None, max_depth=None, seed_stride=1 << 20):
    """Guided (spp samples, training included) vs plain at the guided render's
    device time, over `seeds` disjoint frame ranges.  Returns a dict."""
    guide = guide if guide is not None else GuideConfig()
    plain = load_scene(scene, flags=FLAGS, max_depth=max_depth)
    _, ms_probe = _render(plain, 8, 0)          # warm-up and per-spp cost
    ms_probe = _render(plain, 32, 0)[1] / 32
    gi = load_scene(scene, flags=FLAGS, max_depth=max_depth)
    out = {"spp_guided": spp, "seeds": seeds, "relmse_guided": [], "relmse_plain": [], "spp_plain": [],
           "ms_guided": [], "ms_plain": [], "train_ms": [], "final_loss": []}
    for k in range(seeds):
        f0 = (k + 1) * seed_stride
        gi.setGuiding(guide)                    # fresh network, trained online in this render
        img_g, ms_g = _render(gi, spp, f0)
        gs = gi.guideStats()
        n_p = max(1, int(round(ms_g / ms_probe)))
        img_p, ms_p = _render(plain, n_p, f0)
        out["relmse_guided"].append(relmse(img_g, ref))
        out["relmse_plain"].append(relmse(img_p, ref))
        out["spp_plain"].append(n_p)
        out["ms_guided"].append(ms_g)
        out["ms_plain"].append(ms_p)
        out["train_ms"].append(gs["ms_train"])
        out["final_loss"].append(gs["last_loss"])
    gi.close()
    plain.close()
    rg, rp = float(np.mean(out["relmse_guided"])), float(np.mean(out["relmse_plain"]))
    out.update({"relmse_guided_mean": rg, "relmse_plain_mean": rp, "plain_over_guided": rp / rg,
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
