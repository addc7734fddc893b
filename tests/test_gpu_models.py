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


@pytest.mark.parametrize("prec,tol", [(ks.KS_FP64, 1e-10), (ks.KS_MIXED, 1e-4), (ks.KS_MIXED_GEO64, 1e-4)])
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
    for prec in (ks.KS_FP64, ks.KS_MIXED, ks.KS_MIXED_GEO64):
        out = np.asarray(ks.render(cache, ks.PolarizedSplats(p), [0.0], [230e9], c["L"], nmax=nmax, slab=0.0, precision=prec))[0, 0]
        errs[prec] = rel_l2(out, ref)
    print("winding", nmax, errs)
    # both mixed marches (FP32 with the FP64 polar state, and FP64) under the FP32 transport: 1e-4
    assert errs[ks.KS_FP64] < 1e-10 and errs[ks.KS_MIXED] < 1e-4 and errs[ks.KS_MIXED_GEO64] < 1e-4, errs


@pytest.mark.parametrize("prec,tol", [(ks.KS_FP64, 1e-10), (ks.KS_MIXED, 1e-4)])
def test_knot_splats_match_oracle(oracle, prec, tol):
    # KnotSplats (trajectories.jl:80-129): centres interpolated between trajectory knots at each
    # emission time, beside pattern-rotating thermal splats; two frames, two frequencies
    a, tho = 0.94, np.deg2rad(163.0)
    rng = np.random.Generator(np.random.PCG64(32))
    pk = scenes.thermal_params(rng, 4, a, rlo=3.0, rhi=7.0)
    pk[3:6] = np.log(rng.uniform(0.8, 2.0, (3, 4)))
    ktimes = np.array([-80.0, -30.0, 20.0, 60.0])
    knots = scenes.trajectory_knots(pk, a, ktimes)
    pt = scenes.thermal_params(rng, 3, a)
    model = ks.CompositeModel(ks.KnotSplats(pk, knots, ktimes), ks.PolarizedSplats(pt))
    cam = ks.Camera((-12.0, 12.0), (-12.0, 12.0), 16)
    cache = ks.GeodesicCache(cam, 96)
    ks.regenerate(cache, a, tho)
    L = ks.gravitational_radius(4e6)
    times, nus = [0.0, 20.0], [230e9, 690e9]
    out = np.asarray(ks.render(cache, model, times, nus, L, precision=prec))
    sets = [("knot", pk, None, knots, ktimes), ("thermal", pt, None)]
    errs = {}
    for v, nu in enumerate(nus):
        for f, t in enumerate(times):
            ref = oracle.polarized_image(a, tho, cam.alpha, cam.beta, 96, 64, sets, t, nu, L)
            assert np.abs(ref).max() > 0
            errs[(nu, t)] = rel_l2(out[v, f], ref)
    # the knot splats alone are seen (their rows 1-3 are not used: moving them changes nothing)
    pk2 = pk.copy()
    pk2[0:3] += 50.0
    out2 = np.asarray(ks.render(cache, ks.CompositeModel(ks.KnotSplats(pk2, knots, ktimes), ks.PolarizedSplats(pt)), times, nus, L,
                                precision=prec))
    print("knots", prec, errs)
    assert max(errs.values()) < tol, errs
    assert np.array_equal(out, out2)


@pytest.mark.parametrize("prec,tol", [(ks.KS_FP64, 1e-10), (ks.KS_MIXED, 1e-4)])
def test_uneven_sample_counts_match_oracle(oracle, prec, tol):
    # every ray marched with its own N_j = clamp(64 ceil(768 tau_j / 64), 64, 256): identical to a
    # uniform run at N = N_j for that ray (the reference's tiles, cache.jl:241-246)
    c = scenes.config2(res=16, N=256)
    rng = np.random.Generator(np.random.PCG64(33))
    p = scenes.thermal_params(rng, 6, c["a"], rlo=3.0, rhi=9.0)
    cam = ks.Camera((-14.0, 14.0), (-14.0, 14.0), 16)
    cache = ks.GeodesicCache(cam, 256)
    ks.regenerate(cache, c["a"], c["theta_o"], uneven=(768.0, 64))
    nsorted = cache.nsamples_per_ray
    nscreen = np.empty_like(nsorted)
    nscreen[cache.perm] = nsorted
    counts = np.unique(nscreen)
    assert counts.size >= 2 and counts.min() >= 64 and counts.max() <= 256
    times, nus = [0.0], [86e9, 345e9]
    out = np.asarray(ks.render(cache, ks.PolarizedSplats(p), times, nus, c["L"], precision=prec))
    errs = {}
    for v, nu in enumerate(nus):
        ref = np.zeros((cam.npix, 4))
        for Nj in counts:
            m = nscreen == Nj
            ref[m] = oracle.polarized_image(c["a"], c["theta_o"], cam.alpha[m], cam.beta[m], int(Nj), 64, [("thermal", p, None)], 0.0, nu,
                                            c["L"])
        errs[nu] = rel_l2(out[v, 0], ref)
    # the sample count the metric uses
    cache.count_events(True)
    ks.render(cache, ks.PolarizedSplats(p), times, nus, c["L"], precision=prec)
    ev = cache.event_counts()
    cache.count_events(False)
    print("uneven", prec, counts, errs, ev["samples"], int(nsorted.sum()) * len(nus))
    assert max(errs.values()) < tol, errs
    assert ev["samples"] == int(nsorted.sum()) * len(nus)


def test_autotune_keeps_results(oracle):
    # ks_autotune picks a launch shape by timing; the image stays within the mixed tolerance
    c = scenes.config2(res=24, N=128)
    rng = np.random.Generator(np.random.PCG64(34))
    p = scenes.thermal_params(rng, 8, c["a"])
    cache = ks.GeodesicCache(c["camera"], c["N"])
    ks.regenerate(cache, c["a"], c["theta_o"])
    m = ks.PolarizedSplats(p)
    block, units, ms = ks.autotune(cache, m, [0.0], c["nus"], c["L"], trials=1)
    assert block in (128, 256, 384) and units in (2, 4, 8, 16) and ms > 0
    out = np.asarray(ks.render(cache, m, [0.0], c["nus"], c["L"], precision=ks.KS_MIXED))
    ref = np.asarray(ks.render(cache, m, [0.0], c["nus"], c["L"], precision=ks.KS_FP64))
    assert rel_l2(out, ref) < 1e-4


def test_render_graph_replays_and_follows_parameters():
    """ks_render_graph_capture / ks_graph_launch: a mixed render of device-resident thermal and
    power-law sets captured as a CUDA graph replays to the image of ks_render bit for bit, and after
    an in-place change of the model's parameter buffer the replay equals the re-render; a regenerate
    drops the graph."""
    import torch
    a, tho = 0.94, np.deg2rad(163.0)
    rng = np.random.Generator(np.random.PCG64(35))
    pt = scenes.thermal_params(rng, 6, a)
    pp = scenes.powerlaw_params(rng, 4, a)
    model = ks.CompositeModel(ks.PolarizedSplats(torch.tensor(pt, device="cuda")), ks.PowerLawSplats(torch.tensor(pp, device="cuda")))
    cam = ks.Camera((-12.0, 12.0), (-12.0, 12.0), 16)
    cache = ks.GeodesicCache(cam, 96)
    ks.regenerate(cache, a, tho)
    L = ks.gravitational_radius(4e6)
    times, nus = [0.0, 10.0], [230e9, 345e9]
    g = ks.capture_render(cache, model, times, nus, L)
    ref = ks.render(cache, model, times, nus, L, precision=ks.KS_MIXED).cpu().numpy()
    assert np.abs(ref).max() > 0
    assert np.array_equal(g.replay().cpu().numpy(), ref)
    model.sets()[0].params[:, 12] += np.log(1.5)   # the thermal log densities, in place
    ref2 = ks.render(cache, model, times, nus, L, precision=ks.KS_MIXED).cpu().numpy()
    assert not np.array_equal(ref2, ref)
    assert np.array_equal(g.replay().cpu().numpy(), ref2)
    ks.regenerate(cache, a, tho)
    with pytest.raises(ValueError, match="no captured graph"):
        g.replay()


def test_staging_wait_runs_out_cleanly():
    """The bounded wait of the splat-table staging: with the test hook the barrier is armed but no
    copy is issued, so every block's wait runs out; the kernels record it and return, the call fails
    with KS_ERR_TIMEOUT, and the same context then renders the same image as before (no GPU fault)."""
    c = scenes.config2(res=16, N=64)
    rng = np.random.Generator(np.random.PCG64(36))
    p = scenes.thermal_params(rng, 5, c["a"])
    cache = ks.GeodesicCache(c["camera"], c["N"])
    ks.regenerate(cache, c["a"], c["theta_o"])
    m = ks.PolarizedSplats(p)
    ref = np.asarray(ks.render(cache, m, [0.0], [230e9], c["L"], precision=ks.KS_MIXED))
    cache.set_stage_test(True)
    with pytest.raises(ks.KsError) as err:
        ks.render(cache, m, [0.0], [230e9], c["L"], precision=ks.KS_MIXED)
    assert err.value.status == ks._lib.KS_ERR_TIMEOUT
    cache.set_stage_test(False)
    again = np.asarray(ks.render(cache, m, [0.0], [230e9], c["L"], precision=ks.KS_MIXED))
    assert np.array_equal(again, ref)
