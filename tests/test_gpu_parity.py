"""CUDA path vs the CPU oracle on identical seeded inputs (the parity gate).

FP64 plain path: 1e-10 relative per-pixel Stokes L2 (the bar the reference's Recurrence(64)
output is held to); MIXED path: 1e-4 relative. Sizes are small enough for the oracle to finish in
seconds.
"""
import numpy as np
import pytest

import kerrsplat_b200 as ks
from kerrsplat_b200 import scenes

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
MIXED_TOL = 1e-4


def rel_l2(x, y):
    x, y = np.asarray(x), np.asarray(y)
    return np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300)


def small_cfg1(res=32, N=128):
    c = scenes.config1(res=res, N=N)
    return c


@pytest.fixture(scope="module")
def cfg1_cache():
    c = small_cfg1()
    cache = ks.GeodesicCache(c["camera"], c["N"])
    ks.regenerate(cache, c["a"], c["theta_o"], marcher=ks.Fused(c["M"]))
    return c, cache


def test_ray_constants_match_oracle(cfg1_cache, oracle):
    c, cache = cfg1_cache
    perm = cache.perm
    got = cache.ray_constants()
    ref = oracle.ray_constants(c["a"], c["theta_o"], c["camera"].alpha, c["camera"].beta)[perm]
    # root counts and the case sort (4, 2, 0; stable in screen order)
    assert np.array_equal(got[:, 2], ref[:, 2])
    nr = ref[:, 2]
    assert np.all(np.diff(-nr) >= 0)
    for key in (4, 2, 0):
        sel = np.where(nr == key)[0]
        assert np.all(np.diff(perm[sel]) > 0)
    fin = np.isfinite(ref)
    assert np.array_equal(fin, np.isfinite(got))
    err = np.abs(got[fin] - ref[fin]) / np.maximum(np.abs(ref[fin]), 1.0)
    assert err.max() < 1e-12


def test_samples_match_oracle(cfg1_cache, oracle):
    c, cache = cfg1_cache
    perm = cache.perm
    s = cache.samples()
    ref = oracle.march_samples(c["a"], c["theta_o"], c["camera"].alpha, c["camera"].beta, c["N"], c["M"])
    for key in ("r", "theta", "phi"):
        got = s[key].T
        want = ref[key][perm]
        assert np.max(np.abs(got - want) / np.maximum(np.abs(want), 1.0)) < 1e-10, key
    t_got, t_ref = s["t"].T, ref["t"][perm]
    assert np.max(np.abs(t_got - t_ref) / np.maximum(np.abs(t_ref), 1.0)) < 1e-10
    assert np.array_equal(s["flags"].T, ref["flags"][perm])
    rt, rp = cache.residuals()
    assert np.max(np.abs(rt - ref["resid_t"][perm])) < 1e-10
    assert np.max(np.abs(rp - ref["resid_phi"][perm])) < 1e-10
    assert np.max(rt) < 1e-6 and np.max(rp) < 1e-6


def test_thin_image_fp64_and_mixed(cfg1_cache, oracle):
    c, cache = cfg1_cache
    ref = oracle.thin_image(c["a"], c["theta_o"], c["camera"].alpha, c["camera"].beta, c["N"], c["M"], c["params"], c["t_obs"])
    img64 = ks.thin_image(cache, c["params"], c["t_obs"], precision=ks.KS_FP64)
    got64 = np.asarray(img64).T.ravel()
    assert rel_l2(got64, ref) < FP64_TOL
    img32 = ks.thin_image(cache, c["params"], c["t_obs"], precision=ks.KS_MIXED)
    got32 = np.asarray(img32).T.ravel()
    assert rel_l2(got32, ref) < MIXED_TOL


@pytest.fixture(scope="module")
def cfg2_small():
    c = scenes.config2(res=24, N=128)
    rng = np.random.Generator(np.random.PCG64(11))
    p = scenes.thermal_params(rng, 8, c["a"])
    c["params"] = p
    cache = ks.GeodesicCache(c["camera"], c["N"])
    ks.regenerate(cache, c["a"], c["theta_o"], marcher=ks.Fused(c["M"]))
    return c, cache


def test_polarized_fp64_matches_oracle(cfg2_small, oracle):
    c, cache = cfg2_small
    cam = c["camera"]
    out = np.asarray(ks.render(cache, ks.PolarizedSplats(c["params"]), [0.0], c["nus"], c["L"], precision=ks.KS_FP64))
    for f, nu in enumerate(c["nus"]):
        ref = oracle.polarized_image(c["a"], c["theta_o"], cam.alpha, cam.beta, c["N"], c["M"], [("thermal", c["params"], None)], 0.0, nu, c["L"])
        assert np.abs(ref).max() > 0
        err = np.linalg.norm(out[f, 0] - ref, axis=1) / np.maximum(np.linalg.norm(ref, axis=1), 1e-300)
        tot = rel_l2(out[f, 0], ref)
        assert tot < FP64_TOL, (nu, tot)
        bright = np.linalg.norm(ref, axis=1) > 1e-6 * np.linalg.norm(ref, axis=1).max()
        assert err[bright].max() < 1e-8, (nu, err[bright].max())


def test_polarized_mixed_within_1e4(cfg2_small, oracle):
    c, cache = cfg2_small
    cam = c["camera"]
    out = np.asarray(ks.render(cache, ks.PolarizedSplats(c["params"]), [0.0], c["nus"], c["L"], precision=ks.KS_MIXED))
    errs = {}
    for f, nu in enumerate(c["nus"]):
        ref = oracle.polarized_image(c["a"], c["theta_o"], cam.alpha, cam.beta, c["N"], c["M"], [("thermal", c["params"], None)], 0.0, nu, c["L"])
        # per-pixel relative Stokes L2, and each Stokes image's relative L2
        pix = np.linalg.norm(out[f, 0] - ref, axis=1) / np.maximum(np.linalg.norm(ref, axis=1), 1e-300)
        bright = np.linalg.norm(ref, axis=1) > 1e-3 * np.linalg.norm(ref, axis=1).max()
        errs[nu] = (rel_l2(out[f, 0], ref), [rel_l2(out[f, 0, :, q], ref[:, q]) for q in range(4)], pix[bright].max())
    print("mixed vs FP64 oracle (total, per Stokes, worst bright pixel):", errs)
    for nu, (tot, per, worst) in errs.items():
        assert tot < MIXED_TOL, (nu, tot)
        assert per[0] < MIXED_TOL, (nu, per)


def test_render_before_regenerate_raises():
    c = small_cfg1(res=8, N=16)
    cache = ks.GeodesicCache(c["camera"], c["N"])
    with pytest.raises(ks.KsError):
        ks.thin_image(cache, c["params"], 0.0)
    with pytest.raises(ValueError):
        ks.regenerate(cache, 1.5, 0.3)
