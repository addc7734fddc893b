"""GPU parity of the other consumers of ks_render against the oracle: a composite of thermal,
power-law and kappa splat sets (transport.jl:348-358, populations.jl) over two frames and two
frequencies, and the half-orbit truncation (nmax, transport.jl:182-188)."""
import numpy as np
import pytest

import kerrsplat_b200 as ks
from kerrsplat_b200 import scenes

pytestmark = pytest.mark.gpu


def rel_l2(x, y):
    return np.linalg.norm(np.asarray(x) - np.asarray(y)) / max(np.linalg.norm(y), 1e-300)


@pytest.fixture(scope="module")
def composite():
    a, tho = 0.94, np.deg2rad(163.0)
    rng = np.random.Generator(np.random.PCG64(31))
    pt = scenes.thermal_params(rng, 4, a)
    pp = scenes.powerlaw_params(rng, 4, a)
    pk = scenes.kappa_params(rng, 4, a)
    kap = ks.KappaSplats(pk)
    model = ks.CompositeModel(ks.PolarizedSplats(pt), ks.PowerLawSplats(pp), kap)
    cam = ks.Camera((-12.0, 12.0), (-12.0, 12.0), 20)
    cache = ks.GeodesicCache(cam, 96)
    ks.regenerate(cache, a, tho)
    sets = [("thermal", pt, None), ("powerlaw", pp, None), ("kappa", pk, kap.hyp)]
    return dict(a=a, tho=tho, cam=cam, cache=cache, model=model, sets=sets, L=ks.gravitational_radius(4e6),
                times=[0.0, 10.0], nus=[230e9, 690e9])


@pytest.mark.parametrize("prec,tol", [(ks.KS_FP64, 1e-10), (ks.KS_MIXED, 1e-4), (ks.KS_MIXED_FP32, 1e-3)])
def test_composite_cube_matches_oracle(composite, oracle, prec, tol):
    c = composite
    out = np.asarray(ks.render(c["cache"], c["model"], c["times"], c["nus"], c["L"], precision=prec))
    errs = {}
    for v, nu in enumerate(c["nus"]):
        for f, t in enumerate(c["times"]):
            ref = oracle.polarized_image(c["a"], c["tho"], c["cam"].alpha, c["cam"].beta, 96, 64, c["sets"], t, nu, c["L"])
            assert np.abs(ref).max() > 0
            errs[(nu, t)] = rel_l2(out[v, f], ref)
    print("composite", prec, errs)
    assert max(errs.values()) < tol, (prec, errs)


@pytest.mark.parametrize("nmax", [0, 1])
def test_winding_truncation_matches_oracle(oracle, nmax):
    c = scenes.config2(res=16, N=128)
    rng = np.random.Generator(np.random.PCG64(8))
    p = scenes.thermal_params(rng, 6, c["a"])
    cache = ks.GeodesicCache(c["camera"], c["N"])
    ks.regenerate(cache, c["a"], c["theta_o"])
    ref = oracle.polarized_image(c["a"], c["theta_o"], c["camera"].alpha, c["camera"].beta, c["N"], c["M"], [("thermal", p, None)],
                                 0.0, 230e9, c["L"], nmax=nmax, slab=0.0)
    errs = {}
    for prec in (ks.KS_FP64, ks.KS_MIXED, ks.KS_MIXED_FP32):
        out = np.asarray(ks.render(cache, ks.PolarizedSplats(p), [0.0], [230e9], c["L"], nmax=nmax, slab=0.0, precision=prec))[0, 0]
        errs[prec] = rel_l2(out, ref)
    print("winding", nmax, errs)
    # the all-FP32 march is held to 1e-3: its error comes from the march (axis-grazing rays), not the transport
    assert errs[ks.KS_FP64] < 1e-10 and errs[ks.KS_MIXED] < 1e-4 and errs[ks.KS_MIXED_FP32] < 1e-3, errs
