"""Helpers for the GPU parity tests: batch calls of the cl_unit_* entry points
(the device functions the integrator runs) and ulp-level comparisons.

Tolerance (the target is 4 ulp in FP32 against the reference's functions):
* scalars: distance in units in the last place of the value;
* vectors (directions, colours): per-row maximum component error in ulps of
  the row's magnitude (max |component|), since a unit vector's near-zero
  components carry the absolute error of the whole vector;
* values beyond 4 ulp are accepted only when explained: the FP64 evaluation
  of the same formula shows that the FP32 formula is ill-conditioned there
  (the GPU is no farther from FP64 than `slack` times the CPU FP32 value is),
  or the input is flagged ill-conditioned (warp rim, poles, cell boundaries,
  branch decisions within a few ulp).  Unexplained outliers are bounded.
"""
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


def _report(name, err, max_ulp, unexplained, n):
    hist = {k: int(np.sum(err == k)) for k in range(0, max_ulp + 1)}
    hist[f">{max_ulp}"] = int(np.sum(err > max_ulp))
    finite = err[np.isfinite(err)]
    mx = float(finite.max()) if len(finite) else 0.0
    print(f"[ulp] {name}: n={n} max={mx:.0f} within{max_ulp}={np.mean(err <= max_ulp):.6f} hist={hist} "
          f"unexplained={unexplained}")
    return hist


def _finish(name, err, bad_ok, max_ulp, min_frac, max_unexplained_frac):
    n = len(err)
    bad = err > max_ulp
    unexplained = int(np.sum(bad & ~bad_ok))
    _report(name, np.where(np.isfinite(err), np.round(err), np.inf), max_ulp, unexplained, n)
    frac = float(np.mean(~bad))
    assert frac >= min_frac, f"{name}: only {frac:.5f} within {max_ulp} ulp"
    assert unexplained <= max(2, int(max_unexplained_frac * n)), f"{name}: {unexplained} unexplained outliers"


def check_ulp(name, got, ref, max_ulp=4, min_frac=0.999, ref64=None, other=None, ill=None, slack=8.0,
              rel_ok=None, max_unexplained_frac=5e-4, cond_ulp=None):
    """Scalars.  rel_ok: outliers within this relative error of `ref` count as
    explained; cond_ulp: per-value error bound (ulps) from the conditioning."""
    got = np.asarray(got, np.float32).ravel()
    ref = np.asarray(ref, np.float32).ravel()
    err = ulp_diff(got, ref).astype(np.float64)
    ok = np.zeros(len(err), bool)
    if cond_ulp is not None:
        ok |= err <= np.asarray(cond_ulp, np.float64).ravel()
    if ref64 is not None:
        r64 = np.asarray(ref64, np.float64).ravel()
        o = (np.asarray(other, np.float32).ravel() if other is not None else ref).astype(np.float64)
        unit = np.spacing(np.abs(r64).astype(np.float32)).astype(np.float64)
        ok |= np.abs(got - r64) <= slack * np.abs(o - r64) + 4 * unit
        ok |= np.isnan(got) & np.isnan(r64)
    if ill is not None:
        ok |= np.asarray(ill, bool).ravel()
    if rel_ok is not None:
        ok |= np.abs(got.astype(np.float64) - ref) <= rel_ok * np.abs(ref.astype(np.float64))
    _finish(name, err, ok, max_ulp, min_frac, max_unexplained_frac)


def vec_err(got, ref):
    """Per-row max |got - ref| in ulps of max |ref| of the row."""
    g = np.asarray(got, np.float64).reshape(len(got), -1)
    r = np.asarray(ref, np.float64).reshape(len(ref), -1)
    scale = np.max(np.abs(r), axis=1)
    unit = np.spacing(np.maximum(scale, 1e-30).astype(np.float32)).astype(np.float64)
    with np.errstate(invalid="ignore"):
        d = np.abs(g - r)
    nan_g, nan_r = np.isnan(g), np.isnan(r)
    d[nan_g & nan_r] = 0.0
    d[nan_g ^ nan_r] = np.inf
    err = np.max(d, axis=1) / unit
    zero = scale == 0
    err[zero] = np.where(np.max(np.abs(np.nan_to_num(g[zero], nan=1.0)), axis=1) == 0, 0.0, np.inf)
    return err, unit


def check_vec(name, got, ref, max_ulp=4, min_frac=0.999, ref64=None, other=None, ill=None, slack=8.0,
              max_unexplained_frac=5e-4, cond_ulp=None):
    """Vectors (rows).  cond_ulp: per-row error bound (ulps) from the
    conditioning of the formula; rows within it count as explained."""
    err, unit = vec_err(got, ref)
    ok = np.zeros(len(err), bool)
    if cond_ulp is not None:
        ok |= err <= np.asarray(cond_ulp, np.float64).ravel()
    if ref64 is not None:
        g = np.asarray(got, np.float64).reshape(len(got), -1)
        r64 = np.asarray(ref64, np.float64).reshape(len(got), -1)
        o = np.asarray(other if other is not None else ref, np.float64).reshape(len(got), -1)
        with np.errstate(invalid="ignore"):
            eg = np.nanmax(np.abs(g - r64), axis=1)
            eo = np.nanmax(np.abs(o - r64), axis=1)
        ok |= eg <= slack * eo + 4 * unit
    if ill is not None:
        ok |= np.asarray(ill, bool).ravel()
    _finish(name, err, ok, max_ulp, min_frac, max_unexplained_frac)


def bilinear64(tex, u, v):
    """FP64 evaluation of the RGBA32F wrap/bilinear lookup (same definition as
    the device and the oracle), for conditioning estimates."""
    h, w = tex.shape[:2]
    t = tex.reshape(h * w, 4).astype(np.float64)
    u = u - np.floor(u); v = v - np.floor(v)
    x = u * w - 0.5; y = v * h - 0.5
    fx, fy = np.floor(x), np.floor(y)
    ax, ay = (x - fx)[:, None], (y - fy)[:, None]
    ix, iy = fx.astype(np.int64), fy.astype(np.int64)
    x0, x1, y0, y1 = ix % w, (ix + 1) % w, iy % h, (iy + 1) % h
    top = t[y0 * w + x0] * (1 - ax) + t[y0 * w + x1] * ax
    bot = t[y1 * w + x0] * (1 - ax) + t[y1 * w + x1] * ax
    return (top * (1 - ay) + bot * ay)[:, :3]
