"""Benchmark: plain wavefront path tracing on one B200 (or N independent replicas).

Workload (cfg2): 1920x1080 image, ~4.7M-triangle scene (1024x1024-vertex fBm
terrain + 512 icosphere/torus meshes), 2048x1024 HDRI dome + directional
light, max depth 8, Russian roulette from depth 3.  One step = one render call
of the configuration's 64-spp frame (64 x 2,073,600 camera paths; within the
call the next iteration's paths start in the slots that finished paths free).
The rate at one iteration per call is reported beside it.  The reference's
estimator (compat flags) with the B200 alias-table dome sampler.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun with N ranks, every rank renders its own replica (the path
tracer does not shard: replicas only); value = all ranks' paths / max time.
`--impl reference` times the reference's algorithm on the host cores (the
CPU oracle port, all threads), rank 0 only.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mpaths/s and equal-time relMSE vs FP64 oracle, neural-guided vs plain, 1 B200"
UNIT = "Mpaths/s"
L2_BYTES = 126 * 1024 * 1024
RAY_IN, HIT_OUT, NODE_BYTES, TRI_BYTES = 32, 16, 80, 48


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=6)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=2)
    ap.add_argument("--spp-per-step", type=int, default=0,
                    help="spp of each step's render call (0 = the configuration's frame, at most 64: 64 for config 2)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="CPU baseline sample size")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--profile", type=int, default=0, metavar="CALLS",
                    help="profiling run for ncu: build the workload, make CALLS render calls, print stage times")
    ap.add_argument("--profile-spp", type=int, default=1,
                    help="iterations per render call of --profile (more than one keeps the waves full)")
    ap.add_argument("--slots", type=int, default=0, help="paths in flight (0 = automatic)")
    ap.add_argument("--two-level", action="store_true",
                    help="two-level scene (one tree per mesh, one over the instances) instead of flattened instances")
    ap.add_argument("--no-relmse", action="store_true", help="skip the guided-vs-plain equal-time relMSE")
    ap.add_argument("--no-edit", action="store_true", help="skip the shape-edit (refit vs rebuild) measurement")
    ap.add_argument("--extended", action="store_true",
                    help="cfg4 radiance cache + guiding and cfg5 (4K, both networks) against FP64 references")
    ap.add_argument("--ext-ref-spp4", type=int, default=65536, help="spp of the cfg4 reference for --extended")
    ap.add_argument("--ext-ref-spp5", type=int, default=2048, help="spp of the cfg5 reference for --extended")
    ap.add_argument("--ext-spp5", type=int, default=256, help="neural spp on cfg5 (training included)")
    ap.add_argument("--profile-nets", choices=["guide", "cache"], default=None,
                    help="short workload for ncu: cfg3 with guiding or cfg4 with the radiance cache, "
                         "2 training spp + 2 spp")
    ap.add_argument("--guide-study", action="store_true",
                    help="guiding variants at equal spp against an FP64 reference (one JSON line): on cfg3 "
                         "guided BSDF classes and selection probabilities; on cfg4/cfg5 the same with the "
                         "radiance cache (see --study-config)")
    ap.add_argument("--cache-study", action="store_true",
                    help="with --guide-study on cfg4/cfg5: radiance-cache training variants (steps, batch, "
                         "learning rate) instead of the guiding variants")
    ap.add_argument("--study-config", type=int, default=3, choices=[3, 4, 5],
                    help="scene of --guide-study (3: guiding alone; 4, 5: radiance cache with and without guiding)")
    ap.add_argument("--relmse-ref-spp", type=int, default=8192, help="spp of the cfg3 FP64 reference image")
    ap.add_argument("--relmse-ref-spp4", type=int, default=8192, help="spp of the cfg4 FP64 reference image")
    ap.add_argument("--relmse-seeds", type=int, default=3)
    ap.add_argument("--relmse-spp", type=int, default=128, help="guided spp (training included)")
    return ap.parse_args()


def run_profile_nets(args):
    """A short render for ncu captures of the network kernels."""
    import colvillea_b200 as cb
    from colvillea_b200 import scenes
    if args.profile_nets == "guide":
        s = scenes.config3(0)
        it = cb.load_scene(s, flags=cb.DOME_ALIAS | cb.FILM_FP64)
        it.setGuiding(cb.GuideConfig(train_spp=2))
    else:
        s = scenes.config4(0)
        it = cb.load_scene(s, flags=cb.DOME_ALIAS | cb.FILM_FP64)
        it.setRadianceCache(cb.RadianceCacheConfig(train_spp=2))
    it.render(2)
    it.render(2)
    print(json.dumps({"profile_nets": args.profile_nets, "last_rays_closest": it.stats()["last_rays_closest"]}))
    it.close()
    return 0


def run_profile(args):
    """A short, bounded run of the same kernels for ncu captures."""
    import colvillea_b200 as cb
    from colvillea_b200 import scenes
    s = scenes.CONFIGS[args.config](0)
    it = cb.load_scene(s, flags=cb.COMPAT_ALL | cb.DOME_ALIAS | cb.PROFILE_STAGES, path_slots=args.slots)
    for _ in range(args.profile):
        it.render(args.profile_spp)
        st = it.stats()
        print(json.dumps({**{k: st[k] for k in ("ms_last_render", "ms_trace", "ms_shade", "ms_shadow", "waves",
                                                "last_rays_closest", "last_rays_shadow")},
                          "wave_rays_closest": it.waveRays()}))
    it.close()
    return 0


def step_spp(s, spp_per_step=0):
    """spp of one bench step's render call: the configured frame (64 for
    config 2), at most 64 (config 5's 256-spp 4K frame would take ~10 s)."""
    return spp_per_step or min(s.spp, 64)


def workload_desc(s, spp_per_step=0):
    n = step_spp(s, spp_per_step)
    return {"workload": f"{s.name}: wavefront path tracing {s.width}x{s.height}, max depth {s.max_depth}, RR from "
                        f"{s.rr_start}, {s.num_triangles} triangles, {s.dome().texels.shape[1]}x"
                        f"{s.dome().texels.shape[0]} HDRI dome + directional light; 1 step = one render call of "
                        f"{n} spp over the image (the configured frame is {s.spp} spp)",
            "image": [s.width, s.height], "triangles": s.num_triangles, "max_depth": s.max_depth,
            "rr_start": s.rr_start, "spp_per_step": n,
            "estimator": "reference (compat pdf, frame and escape flags) + alias dome sampler",
            "l2": "inputs larger than L2 (BVH + scene + film > 126 MB), no flush", "seed": 0}


class Dist:
    """One process per GPU (torchrun's RANK / LOCAL_RANK / WORLD_SIZE).  NCCL
    with CUDA tensors on GPUs; gloo with CPU tensors where CUDA is absent (the
    multi-process tests on CPU).  The job is replicas: no data-path collective,
    only a barrier and the max-over-ranks timing."""

    def __init__(self, gpus, backend=None):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        self.device = None
        if self.world > 1:
            import datetime
            import torch
            import torch.distributed as dist
            backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
            timeout = datetime.timedelta(seconds=300)
            if backend == "nccl":
                torch.cuda.set_device(self.local)
                self.device = torch.device("cuda", self.local)
                dist.init_process_group("nccl", timeout=timeout, device_id=self.device)
            else:
                self.device = torch.device("cpu")
                dist.init_process_group(backend, timeout=timeout)
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x):
        if not self.pg:
            return x
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x):
        if not self.pg:
            return x
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.SUM)
        return float(t.item())

    def job_rate(self, units, ms):
        """Whole-job throughput: the units all ranks processed over the
        slowest rank's time (per second)."""
        return self.sum(units) / (self.max(ms) * 1e-3)

    def close(self):
        if self.pg:
            self.pg.barrier()
            self.pg.destroy_process_group()


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index):
        self.index, self.proc, self.lines = index, None, []

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=lambda: self.lines.extend(self.proc.stdout), daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        self.t.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1])); mx = float(f[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(config=2):
    """Per-ray DRAM bytes of the closest-hit kernel from the committed ncu summary of this config, if any."""
    p = os.path.join(ROOT, "profiles", f"trace_closest_cfg{config}.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("dram_bytes_per_ray")
    return None


def _oracle_rate(o, scene, seconds, threads):
    """Paths per second of the oracle at `threads` host threads over an evenly
    strided pixel sample sized to about `seconds` of work: 1 spp over part of
    the image, or several spp over all of it.  A pass shorter than half the
    target is rescaled from its own time and run again; the last pass is the
    one reported."""
    import numpy as np
    import pyoracle
    npx = scene.width * scene.height
    want, spp = min(npx, 2000 if threads > 1 else 400), 1
    while True:
        pix = np.linspace(0, npx - 1, want).astype(np.uint32)
        t0 = time.perf_counter()
        _, _, cnt = o.render(spp, max_depth=scene.max_depth, rr_start=scene.rr_start, flags=pyoracle.COMPAT_ALL,
                             pixels=pix, threads=threads)
        dt = max(time.perf_counter() - t0, 1e-4)
        if dt >= 0.5 * seconds or (want == npx and spp >= 64):
            break
        paths = int(len(pix) * spp * min(seconds / dt, 1000.0))   # paths for about `seconds` at this pass's rate
        want = min(npx, max(want, paths))
        spp = min(64, max(1, -(-paths // npx)))
    sample = (f"{len(pix)} of {npx} pixels (evenly strided), {spp} spp, {dt:.1f} s; {int(cnt[0])} closest + "
              f"{int(cnt[1])} shadow rays ({(cnt[0] + cnt[1]) / dt / 1e6:.3f} Mrays/s)")
    return round(len(pix) * spp / dt / 1e6, 6), sample


def cpu_baseline(scene, seconds, threads):
    """The oracle (the reference's algorithm restated in C++) on the host cores,
    1 spp over a strided pixel sample of the same workload: all threads, and
    one thread (the two rates of the baseline plan)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    pyoracle.build()
    o = pyoracle.OracleScene(scene.flatten())
    value, sample = _oracle_rate(o, scene, seconds, threads)
    v1, s1 = _oracle_rate(o, scene, min(seconds, 8.0), 1)
    return {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample,
            "single_thread": {"value": v1, "unit": UNIT, "cores": 1, "sample": s1}}


def guided_relmse(args):
    """Second half of the metric: equal-time relMSE of the neural tracers vs
    plain path tracing against FP64-accumulated plain references.
      cfg3: the cfg1 scene at 1920x1080, neural-guided (128 spp including
            online training: one Adam step on 2^18 records after each of the
            first 32 spp);
      cfg4: the caustic scene at 1920x1080, depth 16, neural radiance cache
            (paths end in the cache after 2 bounces, 1/16 training paths,
            one Adam step after each of the first 32 spp)."""
    import colvillea_b200 as cb
    from colvillea_b200 import evaluate, scenes
    rnd = lambda v: [round(x, 6) for x in v] if isinstance(v, list) else (round(v, 6) if isinstance(v, float) else v)
    out = {}
    s3 = scenes.config3(0)
    t0 = time.perf_counter()
    ref3 = evaluate.reference(s3, args.relmse_ref_spp)
    t3 = time.perf_counter() - t0
    guide = cb.GuideConfig()
    r = evaluate.equal_time(s3, ref3, args.relmse_spp, seeds=args.relmse_seeds, guide=guide)
    mlp = evaluate.mlp_throughput(s3, guide)
    peak = None
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        peak = float(json.load(open(p)).get("bf16_tflops", 0)) or None
    out["cfg3_guided"] = {
        "workload": f"cfg3: cfg1 scene (10,242 tris) at {s3.width}x{s3.height}, max depth {s3.max_depth}, RR from "
                    f"{s3.rr_start}; guided {args.relmse_spp} spp incl. training ({guide.train_spp} Adam steps, batch "
                    f"{guide.batch}, lr {guide.learning_rate:g}, BSDF fraction {guide.bsdf_fraction:g}, guided classes "
                    f"mask {guide.class_mask}); plain at the same device time",
        "reference": f"plain, corrected estimator, {args.relmse_ref_spp} spp, FP64 film ({t3:.1f} s)",
        **{k: rnd(v) for k, v in r.items()},
        "mlp": {**{k: rnd(v) for k, v in mlp.items()}, "bf16_peak_tflops": peak,
                "infer_frac_of_peak": round(mlp["infer_tflops"] / peak, 4) if peak and mlp["infer_tflops"] else None}}
    # The best equal-time guiding configuration of the equal-spp study on this scene (bench.py --guide-study):
    # the network guides the rough-dielectric vertices only, sampled with probability 0.2.
    tuned = cb.GuideConfig(class_mask=4, bsdf_fraction=0.8)
    rt = evaluate.equal_time(s3, ref3, args.relmse_spp, seeds=args.relmse_seeds, guide=tuned)
    out["cfg3_guided_tuned"] = {
        "workload": f"cfg3 as above; guided classes mask {tuned.class_mask} (rough dielectric), BSDF fraction "
                    f"{tuned.bsdf_fraction:g}, {tuned.train_spp} Adam steps; plain at the same device time",
        "reference": out["cfg3_guided"]["reference"],
        **{k: rnd(v) for k, v in rt.items()}}
    s4 = scenes.config4(0)
    t0 = time.perf_counter()
    ref4 = evaluate.reference(s4, args.relmse_ref_spp4)
    t4 = time.perf_counter() - t0
    cache = cb.RadianceCacheConfig()
    r4 = evaluate.equal_time(s4, ref4, args.relmse_spp, seeds=args.relmse_seeds, cache=cache)
    out["cfg4_radiance_cache"] = {
        "workload": f"cfg4: cfg1 geometry with 60% rough glass (alpha U[0.01,0.1]), 2048x1024 HDRI with one lobe (peak "
                    f"5000, sigma 0.5 deg), {s4.width}x{s4.height}, max depth {s4.max_depth}; radiance cache "
                    f"{args.relmse_spp} spp incl. training ({cache.train_spp} Adam steps, batch {cache.network.batch}, "
                    f"prefix {cache.prefix_bounces} bounces, 1/{1 << cache.train_log2_fraction} training paths); plain "
                    f"at the same device time",
        "reference": f"plain, corrected estimator, {args.relmse_ref_spp4} spp, FP64 film ({t4:.1f} s)",
        **{k: rnd(v) for k, v in r4.items()}}
    return out


def scene_edit(it, s, args, spp=4):
    """Shape edit of the largest mesh (the terrain): a smooth height change
    of up to 0.5 units, then the BVH refitted or rebuilt; device times and
    the render time of `spp` samples on each tree."""
    import numpy as np
    m = max(range(len(s.meshes)), key=lambda i: len(s.meshes[i].indices))
    p = s.meshes[m].positions.copy()
    p[:, 1] += 0.5 * np.sin(p[:, 0] * 0.7) * np.cos(p[:, 2] * 0.5)
    st0 = it.stats()
    out = {"mesh_triangles": int(len(s.meshes[m].indices)), "triangles": st0["triangles"],
           "sah_before_edit": round(st0["bvh_sah_build"], 3)}
    for mode in ("refit", "rebuild"):
        it.updateVertices(m, p, bvh=mode)
        st = it.stats()
        it.render(1)  # graph re-capture after a rebuild
        ms = 0.0
        for _ in range(spp):
            it.render(1)
            ms += it.stats()["ms_last_render"]
        out[mode] = {"bvh_ms": round(st["ms_bvh_update"], 3), "sah": round(st["bvh_sah"], 3),
                     "render_ms_per_spp": round(ms / spp, 3)}
    out["speedup_refit_vs_rebuild"] = round(out["rebuild"]["bvh_ms"] / max(out["refit"]["bvh_ms"], 1e-6), 1)
    return out


def run_guide_study(args):
    """Equal-spp table of guiding variants (training included): does the
    network lower the error, and where.  cfg3: guiding alone, by guided BSDF
    classes and selection probability.  cfg4, cfg5: the radiance cache alone
    and with guiding variants (the relMSE then includes the cache's bias)."""
    import colvillea_b200 as cb
    from colvillea_b200 import evaluate, scenes
    G, C = cb.GuideConfig, cb.RadianceCacheConfig
    if args.study_config == 3:
        sc, spp, ref_spp = scenes.config3(0), args.relmse_spp, args.relmse_ref_spp
        variants = {
            "guided_all_classes_bsdf_fraction_0.5": G(),
            "guided_all_classes_bsdf_fraction_0.5_indirect_only": G(min_depth=2),
            "guided_all_classes_bsdf_fraction_0.5_64_training_steps": G(train_spp=64),
            "guided_all_classes_learned_selection": G(learn_selection=1),
            "guided_diffuse_conductor_bsdf_fraction_0.5": G(class_mask=3),
            "guided_all_classes_bsdf_fraction_0.8": G(bsdf_fraction=0.8),
            "guided_all_classes_bsdf_fraction_0.8_min_alpha_0.1": G(bsdf_fraction=0.8, min_alpha=0.1),
            "guided_dielectric_only_bsdf_fraction_0.5": G(class_mask=4),
            "guided_dielectric_only_bsdf_fraction_0.8": G(class_mask=4, bsdf_fraction=0.8),
            "guided_dielectric_only_bsdf_fraction_0.9": G(class_mask=4, bsdf_fraction=0.9),
            "guided_dielectric_conductor_bsdf_fraction_0.8": G(class_mask=6, bsdf_fraction=0.8),
        }
        label = "cfg3 (cfg1 scene, 1920x1080, depth 5, RR 3)"
    else:
        sc = scenes.config4(0) if args.study_config == 4 else scenes.config5(0)
        spp = args.relmse_spp if args.study_config == 4 else args.ext_spp5
        ref_spp = args.relmse_ref_spp4 if args.study_config == 4 else args.ext_ref_spp5
        variants = {
            "cache": {"cache": C()},
            "cache_128_training_steps": {"cache": C(train_spp=128)},
            "cache_every_spp_training": {"cache": C(train_spp=spp)},
            "cache_batch_2^20": {"cache": C(network={"batch": 1 << 20})},
            "cache_every_spp_training_lr_3e-3": {"cache": C(train_spp=spp, network={"learning_rate": 3e-3})},
            "cache_every_spp_training_beta2_0.999": {"cache": C(train_spp=spp, network={"beta2": 0.999})},
        } if args.cache_study else {
            "cache": {"cache": C()},
            "cache_guided_all_classes_bsdf_fraction_0.5": {"cache": C(), "guide": G()},
            "cache_guided_diffuse_conductor_bsdf_fraction_0.5": {"cache": C(), "guide": G(class_mask=3)},
            "cache_guided_all_classes_bsdf_fraction_0.5_min_alpha_0.1": {"cache": C(), "guide": G(min_alpha=0.1)},
            "cache_guided_all_classes_bsdf_fraction_0.8": {"cache": C(), "guide": G(bsdf_fraction=0.8)},
            "cache_guided_dielectric_only_bsdf_fraction_0.8": {"cache": C(), "guide": G(class_mask=4,
                                                                                     bsdf_fraction=0.8)},
            "guided_all_classes_bsdf_fraction_0.5": G(),
            "guided_all_classes_bsdf_fraction_0.5_min_alpha_0.1": G(min_alpha=0.1),
        }
        label = (f"cfg{args.study_config} ({sc.width}x{sc.height}, depth {sc.max_depth}, RR {sc.rr_start}, "
                 f"{sc.num_triangles} triangles)")
    t0 = time.perf_counter()
    ref = evaluate.reference(sc, ref_spp)
    t_ref = time.perf_counter() - t0
    rows = evaluate.equal_spp(sc, ref, spp, variants, seeds=args.relmse_seeds)
    rnd = lambda d: {k: (round(v, 6) if isinstance(v, float) else ([round(x, 6) for x in v] if isinstance(v, list)
                                                                    else v)) for k, v in d.items()}
    print(json.dumps({"guide_study": f"{label}, corrected estimator, alias dome sampler; {spp} spp per variant incl. "
                                     f"training; {args.relmse_seeds} seeds; reference {ref_spp} spp FP64 "
                                     f"({t_ref:.1f} s)",
                      "rows": {k: rnd(v) for k, v in rows.items()}}))
    return 0


def run_extended(args):
    """The neural configurations not in the default line (one JSON line):
      cfg4: the caustic scene with the radiance cache plus guiding (library
            defaults and the studies' guiding configuration), and the cache
            alone, at equal time against plain, relMSE and bias against a
            65,536-spp FP64 plain reference;
      cfg5: 3840x2160, depth 16, the instanced terrain scene with guiding and
            the radiance cache both on (library defaults, and the studies'
            configuration): equal-time relMSE against plain (FP64
            reference), and the guiding network's inference throughput."""
    import colvillea_b200 as cb
    from colvillea_b200 import evaluate, scenes
    rnd = lambda v: [round(x, 6) for x in v] if isinstance(v, list) else (round(v, 6) if isinstance(v, float) else v)
    peak = None
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        peak = float(json.load(open(p)).get("bf16_tflops", 0)) or None
    out = {"extended": True}
    s4 = scenes.config4(0)
    t0 = time.perf_counter()
    ref4 = evaluate.reference(s4, args.ext_ref_spp4)
    t4 = time.perf_counter() - t0
    # As specified (guiding with the library's defaults on top of the cache), the cache alone, and the cache with
    # the guiding configuration of the equal-spp studies (rough-dielectric vertices, selection probability 0.2).
    tuned_guide = dict(class_mask=4, bsdf_fraction=0.8)
    for name, g, label in (("cfg4_cache_guided", cb.GuideConfig(), "radiance cache + guiding (defaults)"),
                           ("cfg4_cache", None, "radiance cache"),
                           ("cfg4_cache_guided_tuned", cb.GuideConfig(**tuned_guide),
                            "radiance cache + guiding (rough dielectric only, BSDF fraction 0.8)")):
        r = evaluate.equal_time(s4, ref4, args.relmse_spp, seeds=args.relmse_seeds, guide=g,
                                cache=cb.RadianceCacheConfig())
        out[name] = {"reference": f"plain, corrected estimator, {args.ext_ref_spp4} spp, FP64 film ({t4:.1f} s)",
                     "networks": label, **{k: rnd(v) for k, v in r.items()}}
    s5 = scenes.config5(0)
    t0 = time.perf_counter()
    ref5 = evaluate.reference(s5, args.ext_ref_spp5)
    t5 = time.perf_counter() - t0
    g5 = cb.GuideConfig()
    r5 = evaluate.equal_time(s5, ref5, args.ext_spp5, seeds=args.relmse_seeds, guide=g5, cache=cb.RadianceCacheConfig())
    mlp = evaluate.mlp_throughput(s5, g5)
    out["cfg5_guided_cached"] = {
        "workload": f"cfg5: {s5.width}x{s5.height}, max depth {s5.max_depth}, {s5.num_triangles} triangles "
                    f"({len(s5.instances)} instances), 4096x2048 HDRI + directional; guiding + radiance cache "
                    f"{args.ext_spp5} spp incl. training; plain at the same device time",
        "reference": f"plain, corrected estimator, {args.ext_ref_spp5} spp, FP64 film ({t5:.1f} s)",
        **{k: rnd(v) for k, v in r5.items()},
        "mlp": {**{k: rnd(v) for k, v in mlp.items()}, "bf16_peak_tflops": peak,
                "infer_frac_of_peak": round(mlp["infer_tflops"] / peak, 4) if peak and mlp["infer_tflops"] else None}}
    # Both networks on, configured by the cfg5 studies (bench.py --guide-study [--cache-study] --study-config 5):
    # the cache trained for the first 128 spp, guiding on the rough-dielectric vertices only.
    c5 = cb.RadianceCacheConfig(train_spp=128)
    r5t = evaluate.equal_time(s5, ref5, args.ext_spp5, seeds=args.relmse_seeds, guide=cb.GuideConfig(**tuned_guide),
                              cache=c5)
    out["cfg5_guided_cached_tuned"] = {
        "workload": f"cfg5 as above; radiance cache trained for the first {c5.train_spp} spp, guiding on the rough-"
                    f"dielectric vertices only (BSDF fraction 0.8); plain at the same device time",
        "reference": out["cfg5_guided_cached"]["reference"], **{k: rnd(v) for k, v in r5t.items()}}
    print(json.dumps(out))
    return 0


def run_reference(args):
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    from colvillea_b200 import scenes
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import pyoracle
    pyoracle.build()
    s = scenes.CONFIGS[args.config](0)
    threads = os.cpu_count() or 1
    o = pyoracle.OracleScene(s.flatten())
    npx = s.width * s.height
    # size one step to about one second of host work
    probe = np.arange(0, npx, max(1, npx // 2000), dtype=np.uint32)
    t0 = time.perf_counter()
    o.render(1, max_depth=s.max_depth, rr_start=s.rr_start, flags=pyoracle.COMPAT_ALL, pixels=probe, threads=threads)
    per = max(time.perf_counter() - t0, 1e-4) / len(probe)
    nstep = int(min(npx, max(256, 1.0 / per)))
    total, elapsed = 0, 0.0
    for k in range(args.warmup + args.steps):
        pix = ((np.arange(nstep, dtype=np.int64) * (npx // nstep) + k) % npx).astype(np.uint32)
        t0 = time.perf_counter()
        o.render(1, max_depth=s.max_depth, rr_start=s.rr_start, flags=pyoracle.COMPAT_ALL, pixels=pix,
                 threads=threads, frame0=k)
        dt = time.perf_counter() - t0
        if k >= args.warmup:
            total += nstep
            elapsed += dt
    v = total / elapsed / 1e6
    line = {"metric": METRIC, "value": round(v, 6), "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * elapsed / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_desc(s, args.spp_per_step), "parallelism": "host threads",
            "cpu_baseline": {"value": round(v, 6), "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"each step: 1 spp over {nstep} of {npx} pixels (strided), all host threads"},
            "e2e": {"value": round(v, 6), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.profile:
        return run_profile(args)
    if args.profile_nets:
        return run_profile_nets(args)
    if args.extended:
        return run_extended(args)
    if args.guide_study:
        return run_guide_study(args)
    import numpy as np
    import torch
    dist = Dist(args.gpus)
    torch.cuda.set_device(dist.local)
    import colvillea_b200 as cb
    from colvillea_b200 import build as cbuild, scenes
    if not os.path.exists(os.path.join(ROOT, "colvillea_b200", "libcolvillea_b200.so")):
        cbuild.build()
    s = scenes.CONFIGS[args.config](0)
    W, H = s.width, s.height
    # --two-level: config 5's repeated, transformed meshes as a two-level scene
    # (one tree per mesh, one over the instances) instead of one world-space
    # tree over the flattened instances (the default: faster to trace and to
    # build, 60% more scene memory on config 5).
    two = args.two_level
    flags = cb.COMPAT_ALL | cb.DOME_ALIAS | (cb.TWO_LEVEL if two else 0)
    # The timed integrator runs the product path (waves replayed from a CUDA
    # graph); a second one with per-stage CUDA events (each wave launched and
    # synchronised on its own, about 5% slower) gives the stage times and the
    # traversal kernel's time for the roofline, over the same number of steps.
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    it = cb.load_scene(s, flags=flags, path_slots=args.slots)
    torch.cuda.synchronize()
    scene_mb = (free0 - torch.cuda.mem_get_info()[0]) / 2**20
    st0 = it.stats()

    # A step is one render call of `spp` iterations: the configured frame
    # (64 spp for config 2) by default.  Within a call the persistent
    # scheduler starts the next iteration's paths in the slots that finished
    # paths free, so the waves stay full until the last iteration drains.
    spp = step_spp(s, args.spp_per_step)
    # Traversal counters on the identical ray set of the first timed step.
    sit = cb.load_scene(s, flags=flags | cb.TRACE_STATS)
    for _ in range(args.warmup):
        sit.render(spp)
    sit.render(spp)
    sst = sit.stats()
    sit.close()

    for _ in range(args.warmup):
        it.render(spp)
    dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(dist.local)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    ms_dev = 0.0
    rays_c = rays_s = 0
    launches = 0
    for _ in range(args.steps):
        it.render(spp)
        st = it.stats()
        ms_dev += st["ms_last_render"]
        rays_c += st["last_rays_closest"]; rays_s += st["last_rays_shadow"]
        # kRaygen, then per wave: kTraceClosest, kClassifyHits (flattened scenes), 4 x kShade, kTraceShadow,
        # kShadowResolve, kAdvance
        launches += 1 + (8 if two else 9) * st["waves"]
    ev1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    dist.barrier()
    ms_rank = ev0.elapsed_time(ev1)
    # For comparison: one iteration per render call (the reference's render()
    # granularity), where every call ends with its waves draining.
    n1 = 32
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    it.render(1)
    e0.record()
    for _ in range(n1):
        it.render(1)
    e1.record()
    torch.cuda.synchronize()
    value_1spp = dist.job_rate(W * H * n1, e0.elapsed_time(e1)) / 1e6

    # Stage times (CUDA events on the integrator's stream) over the same steps.
    pit = cb.load_scene(s, flags=flags | cb.PROFILE_STAGES, path_slots=args.slots)
    for _ in range(args.warmup):
        pit.render(spp)
    ms_trace = ms_shade = ms_shadow = 0.0
    prays_c = 0
    trace_launches = 0
    for _ in range(args.steps):
        pit.render(spp)
        st = pit.stats()
        ms_trace += st["ms_trace"]; ms_shade += st["ms_shade"]; ms_shadow += st["ms_shadow"]
        prays_c += st["last_rays_closest"]
        trace_launches += st["waves"]
    pit.close()
    value = dist.job_rate(W * H * spp * args.steps, ms_rank) / 1e6
    mrays = dist.job_rate(rays_c + rays_s, ms_rank) / 1e6
    ms = dist.max(ms_rank)

    # End to end through the public API: camera in (host), render, film out to pinned host memory.
    e2e = None
    if not args.no_e2e:
        film = torch.empty((H, W, 4), dtype=torch.float32, pin_memory=True)
        arr = film.numpy()
        cam = np.ascontiguousarray(s.camera, np.float32)
        for _ in range(args.warmup):
            it.updateCamera(cam); it.render(spp); it.readbackFramebufferAsync(arr)
        it.readbackWait()
        dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            it.updateCamera(cam)
            it.render(spp)
            it.readbackFramebufferAsync(arr)   # step k's copy overlaps step k+1's render
        it.readbackWait()
        e1.record()
        torch.cuda.synchronize()
        ems_rank = e0.elapsed_time(e1)
        e2e_value = dist.job_rate(W * H * spp * args.steps, ems_rank) / 1e6
        ems = dist.max(ems_rank)
        e2e = {"value": round(e2e_value, 4), "unit": UNIT,
               "h2d_bytes_per_step": int(cam.nbytes), "d2h_bytes_per_step": int(arr.nbytes),
               "ms_per_step": round(ems / args.steps, 3),
               "pipeline": "camera H2D, render, film mean resolved on the device and copied to pinned host memory "
                           "on a copy stream (cl_readback_film_async); each step's copy overlaps the next render, "
                           "the last one is waited for inside the timed region"}
    edit = scene_edit(it, s, args) if dist.world == 1 and not args.no_edit else None
    it.close()

    if dist.rank != 0:
        dist.close()
        return 0
    # Roofline of the dominant kernel: closest-hit traversal.
    n_rays = max(1, sst["last_rays_closest"])
    nodes_per_ray = sst["trace_nodes"] / n_rays
    tris_per_ray = sst["trace_tris"] / n_rays
    bytes_per_ray = RAY_IN + HIT_OUT + NODE_BYTES * nodes_per_ray + TRI_BYTES * tris_per_ray
    achieved = bytes_per_ray * prays_c / (ms_trace * 1e-3) / 1e9 if ms_trace > 0 else None
    peak, peak_kind = peaks()
    traffic = ncu_traffic(args.config)
    line = {
        "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": dist.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_desc(s, spp),
        "parallelism": f"replicas x{dist.world}" if dist.world > 1 else "single GPU",
        "mrays_per_s": round(mrays, 2),
        "value_1spp_per_call": round(value_1spp, 2),
        "stage_ms_per_spp": {"trace": round(ms_trace / (args.steps * spp), 3),
                             "shade": round(ms_shade / (args.steps * spp), 3),
                             "shadow": round(ms_shadow / (args.steps * spp), 3),
                             "device_total": round(ms_dev / (args.steps * spp), 3)},
        "roofline": {"kernel": "kTraceClosest (8-wide BVH closest hit)", "bound": "hbm",
                     "achieved": round(achieved, 1) if achieved else None, "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4) if achieved else None,
                     "peak_kind": f"{peak_kind} HBM copy",
                     "traffic": round(traffic * prays_c / max(1, trace_launches)) if traffic else None,
                     "bytes_per_ray": round(bytes_per_ray, 1), "nodes_per_ray": round(nodes_per_ray, 2),
                     "tris_per_ray": round(tris_per_ray, 2),
                     "formula": "per closest-hit ray: 32 B ray + 16 B hit + 80 B x nodes + 48 B x triangles",
                     "timing": "kTraceClosest's CUDA-event time on its stream, in a stage-profiled pass of the "
                               "same steps"},
        "clocks": clk, "gpu_launches": launches,
        # The first build of the process (cold: module loading, first allocations) and the second
        # (the traversal-counter integrator's build of the same scene).
        "build": {"bvh_ms": round(st0["ms_bvh_build"], 2), "bvh_ms_cold_wall": round(st0["ms_bvh_build_wall"], 2),
                  "bvh_ms_cold_alloc": round(st0["ms_bvh_build_alloc"], 2),
                  "bvh_ms_warm": round(sst["ms_bvh_build"], 2), "bvh_ms_warm_wall": round(sst["ms_bvh_build_wall"], 2),
                  "bvh_ms_warm_alloc": round(sst["ms_bvh_build_alloc"], 2), "bvh_nodes": st0["bvh_nodes"],
                  "bvh_depth": st0["bvh_depth"], "dome_ms": round(st0["ms_dome_build"], 2),
                  "instancing": "two-level (one tree per mesh + instance tree)" if two else "flattened (one tree)",
                  "scene_device_mb": round(scene_mb, 1)},
    }
    if e2e:
        line["e2e"] = e2e
    if edit:
        line["scene_edit"] = edit
    if dist.world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(s, args.cpu_seconds, os.cpu_count() or 1)
    if dist.world == 1 and not args.no_relmse:
        line["relmse"] = guided_relmse(args)
    print(json.dumps(line))
    dist.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
