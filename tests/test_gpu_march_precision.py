"""The FP32 march of the mixed path (KS_MIXED) against the FP64 march under the same FP32 transport
(KS_MIXED_GEO64), on the two scenes that decided its design:

* configuration 2's scene at 128 x 128, N = 1024: the samples next to a polar turning point in the
  polar cap sit on krang_visible's boundary (recurrence.jl:299-308), so an FP32 cos theta flips their
  validity. That cost 2.6e-4 of the configuration-2 image when the whole march ran in FP32. With the
  polar state in FP64 the flags are the FP64 march's.
* a 16 x 16, N = 128 scene (coarse Mino steps): FP32 Jacobi recurrences and running sums drift between
  anchors (6e-4 at M = 64, shrinking with the anchor spacing). With the radial state and the sums in
  FP64 the drift is gone.

Both hold the FP32 march to 2e-5 relative L2 of the FP64-march image (measured 2.4e-6 and 7.2e-6). The
mixed path's budget against FP64 is 1e-4."""
import numpy as np
import pytest

import kerrsplat_b200 as ks
from kerrsplat_b200 import scenes

pytestmark = pytest.mark.gpu


def rel_l2(x, y):
    return float(np.linalg.norm(x - y) / np.linalg.norm(y))


def test_fp32_march_flags_at_the_polar_turning_points():
    c = scenes.config2(res=128, N=1024)
    cache = ks.GeodesicCache(c["camera"], c["N"])
    ks.regenerate(cache, c["a"], c["theta_o"])
    m = ks.PolarizedSplats(c["params"])
    geo = np.asarray(ks.render(cache, m, [c["t_obs"]], c["nus"], c["L"], precision=ks.KS_MIXED_GEO64))
    f32 = np.asarray(ks.render(cache, m, [c["t_obs"]], c["nus"], c["L"], precision=ks.KS_MIXED))
    errs = [rel_l2(f32[v], geo[v]) for v in range(len(c["nus"]))]
    print("FP32 march vs FP64 march, config-2 scene at 128^2:", errs)
    assert max(errs) < 2e-5, errs
    cache.close()


@pytest.mark.parametrize("M", [64, 16])
def test_fp32_march_does_not_drift_between_anchors(M):
    c = scenes.config2(res=16, N=128)
    rng = np.random.Generator(np.random.PCG64(8))
    p = scenes.thermal_params(rng, 6, c["a"])
    cache = ks.GeodesicCache(c["camera"], c["N"])
    ks.regenerate(cache, c["a"], c["theta_o"], marcher=ks.Fused(M))
    m = ks.PolarizedSplats(p)
    geo = np.asarray(ks.render(cache, m, [0.0], [230e9], c["L"], nmax=0, slab=0.0, precision=ks.KS_MIXED_GEO64))
    f32 = np.asarray(ks.render(cache, m, [0.0], [230e9], c["L"], nmax=0, slab=0.0, precision=ks.KS_MIXED))
    e = rel_l2(f32, geo)
    print("FP32 march vs FP64 march, 16^2 N = 128, M =", M, ":", e)
    assert e < 2e-5, e
    cache.close()
