"""The allocation-free thin image (ks_thin_image_noalloc), for callers whose device memory is owned
by their own allocator and cannot let the library call cudaMalloc (see include/kerrsplat_b200.h).

This file sorts last so that a `-x` run has already run every other test if it fails. The test calls
the new entry point through the C ABI twice in a row (different splat sets, so a stale table from the
first call would show in the second) and compares each image with the existing entry point's, within
the tolerance of the other parity tests (relative L2 1e-10 for FP64, 1e-4 for the FP32 mixed path,
whose two kernels may round differently). It runs alone or after the others.
"""
import ctypes

import numpy as np
import pytest

import kerrsplat_b200 as ks
from kerrsplat_b200 import _lib, scenes

pytestmark = pytest.mark.gpu


def rel_l2(x, y):
    return np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300)


def test_noalloc_thin_image_matches_existing_entry_point():
    import torch
    c = scenes.config1(res=24, N=96)
    cache = ks.GeodesicCache(c["camera"], c["N"])
    ks.regenerate(cache, c["a"], c["theta_o"])
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    p_a = c["params"]
    rng = np.random.Generator(np.random.PCG64(17))
    p_b = p_a[:, :7].copy()
    p_b[12] += rng.uniform(-0.5, 0.5, 7)
    for params in (p_a, p_b):       # two calls in a row
        for prec in (ks.KS_FP64, ks.KS_MIXED):
            for order in (_lib.KS_ORDER_SORTED, _lib.KS_ORDER_SCREEN):
                ref = np.empty(cache.npix)
                buf = np.ascontiguousarray(params.T)
                cache._check(lib.ks_thin_image(cache._ctx, ctypes.c_void_p(buf.ctypes.data), params.shape[1], 0.0, prec,
                                               ctypes.c_void_p(ref.ctypes.data), order))
                p_dev = torch.tensor(buf, device=dev)
                out = torch.full((cache.npix,), float("nan"), dtype=torch.float64, device=dev)
                st = lib.ks_thin_image_noalloc(cache._ctx, ctypes.c_void_p(p_dev.data_ptr()), params.shape[1], 0.0, prec,
                                               ctypes.c_void_p(out.data_ptr()), order)
                assert st == _lib.KS_OK, lib.ks_last_error(cache._ctx)
                got = out.cpu().numpy()
                assert np.all(np.isfinite(got))
                tol = 1e-10 if prec == ks.KS_FP64 else 1e-4
                assert rel_l2(got, ref) < tol, (params.shape[1], prec, order, rel_l2(got, ref))
    # the limit and the pointer kinds are checked before any launch
    too_many = torch.zeros((_lib.KS_NOALLOC_MAX_SPLATS + 1) * 14, dtype=torch.float64, device=dev)
    out = torch.zeros(cache.npix, dtype=torch.float64, device=dev)
    st = lib.ks_thin_image_noalloc(cache._ctx, ctypes.c_void_p(too_many.data_ptr()), _lib.KS_NOALLOC_MAX_SPLATS + 1, 0.0, ks.KS_FP64,
                                   ctypes.c_void_p(out.data_ptr()), _lib.KS_ORDER_SORTED)
    assert st == _lib.KS_ERR_ARGUMENT
    host_out = np.zeros(cache.npix)
    p_dev = torch.tensor(np.ascontiguousarray(p_a.T), device=dev)
    st = lib.ks_thin_image_noalloc(cache._ctx, ctypes.c_void_p(p_dev.data_ptr()), p_a.shape[1], 0.0, ks.KS_FP64,
                                   ctypes.c_void_p(host_out.ctypes.data), _lib.KS_ORDER_SORTED)
    assert st == _lib.KS_ERR_ARGUMENT
    cache.close()


def test_noalloc_wrapper_on_torch_tensors_allocates_no_device_memory():
    """The Python wrapper on CUDA tensors (the transposed parameter copy is made on torch's stream and
    waited for) gives ks_thin_image's image, and a call after the first one leaves the device's free
    memory unchanged (cudaMemGetInfo): the table lives in the static array, the plan and anchors were
    allocated by regenerate."""
    import torch
    c = scenes.config1(res=20, N=80)
    cache = ks.GeodesicCache(c["camera"], c["N"])
    ks.regenerate(cache, c["a"], c["theta_o"])
    dev = torch.device("cuda", 0)
    p = torch.tensor(c["params"], device=dev)
    out = torch.zeros(cache.npix, dtype=torch.float64, device=dev)
    for prec, tol in ((ks.KS_FP64, 1e-10), (ks.KS_MIXED, 1e-4)):
        ref = np.asarray(ks.thin_image_sorted(cache, c["params"], 0.0, precision=prec))
        ks.thin_image_noalloc(cache, p, 0.0, out, precision=prec)       # first call: symbol lookup
        buf = p.t().contiguous()                                           # made before the measurement
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info(dev)
        lib = _lib.load()
        st = lib.ks_thin_image_noalloc(cache._ctx, ctypes.c_void_p(buf.data_ptr()), p.shape[1], 0.0, prec,
                                       ctypes.c_void_p(out.data_ptr()), _lib.KS_ORDER_SORTED)
        assert st == _lib.KS_OK, lib.ks_last_error(cache._ctx)
        free1, _ = torch.cuda.mem_get_info(dev)
        assert free1 == free0, (free0, free1)
        got = out.cpu().numpy()
        assert rel_l2(got, ref) < tol, (prec, rel_l2(got, ref))
    cache.close()
