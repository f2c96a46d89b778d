"""Generates tests/golden/ref_kernels.npz from the reference itself.

Runs the reference's header-only kernel code (BSDFs, GGX, Fresnel, warps,
frames, pcg4d/sampler), compiled on the host from the reference sources by
oracle/ref/Makefile into oracle/_ref/libclref.so, on seeded random inputs and
stores inputs and outputs.  The oracle (oracle/liboracle.so) is pinned against
these vectors by tests/test_oracle_golden.py; the GPU kernels are then checked
against the oracle.

Needs the reference tree, named by the REF environment variable (no default):
    REF=<reference checkout> python tests/golden/gen_golden.py
"""
import ctypes
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libclref.so")
OUT = os.path.join(HERE, "ref_kernels.npz")
N = 2048


def P(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def unit(rng, n, upper=False):
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    if upper:
        v[:, 2] = np.abs(v[:, 2])
    return v.astype(np.float32)


def bsdf_params(rng, n, btype):
    p = np.zeros((n, 11), np.float32)
    p[:, 0:3] = rng.uniform(0.0, 1.0, (n, 3))
    p[:, 3] = rng.uniform(0.002, 0.8, n) if btype else 0.0
    p[:, 4] = rng.uniform(1.05, 2.4, n)
    p[:, 5:8] = rng.uniform(0.05, 2.0, (n, 3))
    p[:, 8:11] = rng.uniform(0.5, 5.0, (n, 3))
    return p


def main():
    ref = os.environ.get("REF")
    if not ref:
        sys.exit("REF is not set: REF=<reference checkout> python tests/golden/gen_golden.py")
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle", "ref"), f"REF={ref}"], check=True)
    L = ctypes.CDLL(REF_LIB)
    rng = np.random.default_rng(20260101)
    g = {}

    # pcg4d and sampler sequences.
    v = rng.integers(0, 2**32, size=(N, 4), dtype=np.uint64).astype(np.uint32)
    v[:16] = np.arange(64, dtype=np.uint32).reshape(16, 4)
    out = np.zeros_like(v)
    L.ref_pcg4d(P(v), P(out), N)
    g["pcg4d_in"], g["pcg4d_out"] = v, out
    seeds = np.stack([rng.integers(0, 3840, N), rng.integers(0, 2160, N), rng.integers(0, 1024, N)], 1).astype(np.uint32)
    seq = np.zeros((N, 8), np.float32)
    L.ref_sampler_sequence(P(seeds), N, 8, P(seq))
    g["sampler_seeds"], g["sampler_seq"] = seeds, seq

    # BSDFs: eval/pdf on directions over the whole sphere, sample on both sides.
    for btype, name in ((0, "diffuse"), (1, "conductor"), (2, "dielectric")):
        p = bsdf_params(rng, N, btype)
        wo = unit(rng, N)
        wi = unit(rng, N)
        # a quarter of the cases in the same upper hemisphere (non-zero lobes)
        q = N // 4
        wo[:q, 2] = np.abs(wo[:q, 2]); wi[:q, 2] = np.abs(wi[:q, 2])
        u2 = rng.uniform(0.0, 1.0, (N, 2)).astype(np.float32)
        ev = np.zeros((N, 3), np.float32); pdf = np.zeros(N, np.float32)
        L.ref_bsdf_eval(btype, P(p), P(wo), P(wi), P(ev), N)
        L.ref_bsdf_pdf(btype, P(p), P(wo), P(wi), P(pdf), N)
        swi = np.zeros((N, 3), np.float32); spdf = np.zeros(N, np.float32); sval = np.zeros((N, 3), np.float32)
        L.ref_bsdf_sample(btype, P(p), P(wo), P(u2), P(swi), P(spdf), P(sval), N)
        g.update({f"{name}_params": p, f"{name}_wo": wo, f"{name}_wi": wi, f"{name}_u2": u2, f"{name}_eval": ev,
                  f"{name}_pdf": pdf, f"{name}_swi": swi, f"{name}_spdf": spdf, f"{name}_sval": sval})

    # GGX.
    alpha = rng.uniform(0.0, 0.9, N).astype(np.float32)
    m = unit(rng, N); wi = unit(rng, N); wo = unit(rng, N)
    D, G1, G, pa = (np.zeros(N, np.float32) for _ in range(4))
    L.ref_ggx_eval(P(alpha), P(m), P(wi), P(wo), P(D), P(G1), P(G), P(pa), N)
    u2 = rng.uniform(0.0, 1.0, (N, 2)).astype(np.float32)
    sm = np.zeros((N, 3), np.float32); sp = np.zeros(N, np.float32)
    L.ref_ggx_sample(P(alpha), P(u2), P(sm), P(sp), N)
    g.update(ggx_alpha=alpha, ggx_m=m, ggx_wi=wi, ggx_wo=wo, ggx_D=D, ggx_G1=G1, ggx_G=G, ggx_pdfAll=pa, ggx_u2=u2,
             ggx_sm=sm, ggx_spdf=sp)

    # Fresnel.
    cosi = rng.uniform(-1.0, 1.0, N).astype(np.float32)
    eta3 = rng.uniform(0.05, 3.0, (N, 3)).astype(np.float32)
    k3 = rng.uniform(0.0, 6.0, (N, 3)).astype(np.float32)
    fc = np.zeros((N, 3), np.float32)
    L.ref_fresnel_conductor(P(cosi), P(eta3), P(k3), P(fc), N)
    eta = rng.uniform(0.5, 2.5, N).astype(np.float32)
    fd = np.zeros(N, np.float32); ct = np.zeros(N, np.float32)
    L.ref_fresnel_dielectric(P(cosi), P(eta), P(fd), P(ct), N)
    g.update(fres_cos=cosi, fres_eta3=eta3, fres_k3=k3, fres_cond=fc, fres_eta=eta, fres_diel=fd, fres_cost=ct)

    # Warps, frames.
    u2 = rng.uniform(0.0, 1.0, (N, 2)).astype(np.float32)
    u2[:4] = [[0.5, 0.5], [0.0, 0.0], [0.999, 0.5], [0.5, 0.25]]
    disk = np.zeros((N, 2), np.float32); hemi = np.zeros((N, 3), np.float32)
    L.ref_warp(P(u2), P(disk), P(hemi), N)
    a = unit(rng, N)
    fb = np.zeros_like(a); fcc = np.zeros_like(a)
    L.ref_make_frame(P(a), P(fb), P(fcc), N)
    s_, t_, n_ = unit(rng, N), unit(rng, N), unit(rng, N)
    vv = unit(rng, N)
    loc = np.zeros_like(vv); wld = np.zeros_like(vv)
    L.ref_frame(P(s_), P(t_), P(n_), P(vv), P(loc), P(wld), N)
    g.update(warp_u2=u2, warp_disk=disk, warp_hemi=hemi, mf_a=a, mf_b=fb, mf_c=fcc, fr_s=s_, fr_t=t_, fr_n=n_, fr_v=vv,
             fr_local=loc, fr_world=wld)

    np.savez_compressed(OUT, **g)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    sys.exit(main())
