"""cl_dome_build_tables_noalloc: the dome preprocessing for callers that cannot
allocate device memory.

Such callers (hosts whose allocator owns all device memory in a pool, render
callbacks that must not allocate) hand in device buffers for the texels and
every table; the function's FP64 scratch is a static device array, so it
calls no allocator.  Here the test plays that caller: it allocates the
buffers itself (with torch) and compares the tables of two calls in a row,
on two different textures, with what the allocating path (cl_build_emitters
+ cl_get_dome_tables) builds for the same texels.  Same kernels and FP64
arithmetic, so the CDF/pdf tables must be bit-identical; the alias tables must
encode the same density.
"""
import ctypes

import numpy as np
import pytest

import colvillea_b200 as cb
from colvillea_b200 import _native as N
from colvillea_b200 import scenes

pytestmark = pytest.mark.gpu


def tables_allocating(tex):
    h, w = tex.shape[:2]
    it = cb.Integrator.createIntegrator(cb.IntegratorType.WavefrontPathTracing, 8, 8)
    it.buildEmitters([scenes.Emitter(scenes.EMIT_DOME, texels=tex)])
    out = it.domeTables(w, h)
    it.close()
    return out


def tables_noalloc(tex):
    import torch
    h, w = tex.shape[:2]
    dev = torch.device("cuda", torch.cuda.current_device())
    t = torch.from_numpy(np.ascontiguousarray(tex, np.float32).reshape(-1)).to(dev)
    pU = torch.full(((w + 1) * h,), -1.0, dtype=torch.float32, device=dev)
    cU = torch.full_like(pU, -1.0)
    pV = torch.full((h + 1,), -1.0, dtype=torch.float32, device=dev)
    cV = torch.full_like(pV, -1.0)
    ar = torch.zeros(2 * h, dtype=torch.int32, device=dev)
    ac = torch.zeros(2 * w * h, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream()
    N.call("cl_dome_build_tables_noalloc", ctypes.c_void_p(t.data_ptr()), w, h, ctypes.c_void_p(pU.data_ptr()),
           ctypes.c_void_p(cU.data_ptr()), ctypes.c_void_p(pV.data_ptr()), ctypes.c_void_p(cV.data_ptr()),
           ctypes.c_void_p(ar.data_ptr()), ctypes.c_void_p(ac.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
    stream.synchronize()
    return [x.cpu().numpy() for x in (pU, cU, pV, cV)], ar.cpu().numpy().view(np.uint32), ac.cpu().numpy().view(np.uint32)


def alias_mass(table, n):
    """Probability mass per bucket encoded by an alias table {prob bits, alias}."""
    prob = table[0::2].view(np.float32).astype(np.float64)
    alias = table[1::2].astype(np.int64)
    assert np.all((prob >= 0) & (prob <= 1)) and np.all((alias >= 0) & (alias < n))
    mass = prob.copy()
    np.add.at(mass, alias, 1.0 - prob)
    return mass / n


def test_noalloc_matches_allocating_path_on_two_calls():
    rng = np.random.default_rng(11)
    textures = [scenes.hdri(512, 256, [(d, 3.0, 40.0) for d in scenes.random_upper_dirs(rng, 3)], rng),
                scenes.hdri(1024, 512, [(d, 1.0, 400.0) for d in scenes.random_upper_dirs(rng, 5)], rng)]
    for k, tex in enumerate(textures):  # the second call reuses the scratch at the maximum size
        h, w = tex.shape[:2]
        ref = tables_allocating(tex)
        got, ar, ac = tables_noalloc(tex)
        for name, a, b in zip(("pUcondV_c", "CDFpUcondV", "pV_c", "CDFpV"), got, ref):
            assert np.array_equal(a, b), f"call {k}: {name} differs"
        f = ref[0].reshape(h, w + 1)[:, :w].astype(np.float64)
        for v in (0, h // 3, h // 2, h - 1):
            np.testing.assert_allclose(alias_mass(ac[2 * w * v: 2 * w * (v + 1)], w), f[v] / f[v].sum(),
                                       rtol=1e-4, atol=1e-9)
        rows = ref[2][:h].astype(np.float64)
        np.testing.assert_allclose(alias_mass(ar, h), rows / rows.sum(), rtol=1e-4, atol=1e-9)


def test_noalloc_rejects_sizes_beyond_the_static_scratch():
    import torch
    buf = torch.zeros(64, dtype=torch.float32, device="cuda")
    p = ctypes.c_void_p(buf.data_ptr())
    L = N.lib()
    assert L.cl_dome_build_tables_noalloc(p, 2048, 1024, p, p, p, p, p, p, None) == N.CL_ERR_INVALID_ARG
    assert "exceeds the static scratch" in N.last_error()
    assert L.cl_dome_build_tables_noalloc(p, 64, 8192, p, p, p, p, p, p, None) == N.CL_ERR_INVALID_ARG
    assert L.cl_dome_build_tables_noalloc(None, 64, 32, p, p, p, p, p, p, None) == N.CL_ERR_INVALID_ARG
