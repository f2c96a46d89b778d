"""Helpers for the GPU parity tests: batch calls of the cl_unit_* entry points
(the device functions the integrator runs) and ulp-level comparisons."""
import ctypes

import numpy as np

from colvillea_b200 import _native as N
from conftest import ulp_diff


def P(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def f32(a):
    return np.ascontiguousarray(a, np.float32)


def gpu_bsdf_eval(t, params, wo, wi):
    out = np.zeros((len(wo), 3), np.float32)
    N.call("cl_unit_bsdf_eval", t, P(f32(params)), P(f32(wo)), P(f32(wi)), P(out), len(wo))
    return out


def gpu_bsdf_pdf(t, params, wo, wi, compat=True):
    out = np.zeros(len(wo), np.float32)
    N.call("cl_unit_bsdf_pdf", t, P(f32(params)), P(f32(wo)), P(f32(wi)), P(out), len(wo), int(compat))
    return out


def gpu_bsdf_sample(t, params, wo, u2):
    n = len(wo)
    wi = np.zeros((n, 3), np.float32); pdf = np.zeros(n, np.float32); v = np.zeros((n, 3), np.float32)
    N.call("cl_unit_bsdf_sample", t, P(f32(params)), P(f32(wo)), P(f32(u2)), P(wi), P(pdf), P(v), n)
    return wi, pdf, v


def check_ulp(name, got, ref, max_ulp=4, min_frac=0.999, ref64=None, other=None, slack=8.0):
    """got vs ref (float32): at least `min_frac` of the values within `max_ulp`;
    the remaining ones, when an FP64 evaluation `ref64` of the same formula is
    given, must be no farther from it than `slack` times the CPU FP32 value
    `other` is (the FP32 formula itself is ill-conditioned there) plus 4 ulp.
    Returns the ulp histogram summary."""
    got = np.asarray(got, np.float32).ravel()
    ref = np.asarray(ref, np.float32).ravel()
    d = ulp_diff(got, ref)
    frac = float(np.mean(d <= max_ulp))
    hist = {k: int(np.sum(d == k)) for k in range(0, max_ulp + 1)}
    hist[f">{max_ulp}"] = int(np.sum(d > max_ulp))
    bad = np.nonzero(d > max_ulp)[0]
    unexplained = len(bad)
    if ref64 is not None and len(bad):
        r64 = np.asarray(ref64, np.float64).ravel()[bad]
        o = (np.asarray(other, np.float32).ravel() if other is not None else ref)[bad].astype(np.float64)
        g = got[bad].astype(np.float64)
        tol = slack * np.abs(o - r64) + 4 * np.spacing(np.abs(r64).astype(np.float32)).astype(np.float64)
        ok = (np.abs(g - r64) <= tol) | (np.isnan(g) & np.isnan(r64))
        unexplained = int(np.sum(~ok))
    print(f"[ulp] {name}: n={len(d)} max={int(d.max()) if len(d) else 0} within{max_ulp}={frac:.6f} "
          f"hist={hist} unexplained={unexplained}")
    assert frac >= min_frac, f"{name}: only {frac:.5f} within {max_ulp} ulp ({hist})"
    if ref64 is not None:
        assert unexplained <= max(2, int(0.0005 * len(d))), f"{name}: {unexplained} outliers not explained by FP64"
    return hist
