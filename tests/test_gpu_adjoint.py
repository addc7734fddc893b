"""GPU parity of the adjoint (the dual sweep, src/Splats/dual_gradient.jl; chi2_gradient!,
src/Fit/Fit.jl:502-577) against central finite differences of the CPU oracle's polarized image, the
check the reference's own gradient gates make (test/test_polarized_splats.jl:318-364; the
reference's Enzyme gradient cannot run here).

Tolerances: the FP64 adjoint against the FD gradient within 1e-5 per parameter (relative, with a
floor of 1e-4 of the largest component; the FD step is 1e-7 relative, so its own error is ~1e-8);
the mixed (FP32 transport) adjoint within 1e-3 of the FP64 adjoint in the relative L2 norm over all
parameters, and per parameter above 1e-2 of the largest component.
"""
import numpy as np
import pytest

import kerrsplat_b200 as ks
from kerrsplat_b200 import scenes

pytestmark = pytest.mark.gpu

NS, RES, N = 5, 10, 64


@pytest.fixture(scope="module")
def scene():
    c = scenes.config2(res=RES, N=N)
    rng = np.random.Generator(np.random.PCG64(21))
    p = scenes.thermal_params(rng, NS, c["a"], rlo=3.0, rhi=8.0)
    # large splats close to the hole so that every one of them is seen by the small screen
    p[3:6] = np.log(rng.uniform(1.0, 2.5, (3, NS)))
    cam = ks.Camera((-10.0, 10.0), (-10.0, 10.0), RES)
    cache = ks.GeodesicCache(cam, N)
    ks.regenerate(cache, c["a"], c["theta_o"])
    times, nus = np.array([0.0, 5.0]), np.array([86e9, 345e9])
    ds = np.random.Generator(np.random.PCG64(22)).standard_normal((len(nus), len(times), cam.npix, 4))
    return dict(c=c, p=p, cam=cam, cache=cache, times=times, nus=nus, ds=ds, N=N)


def oracle_loss(oracle, s, p, nmax=-1, slab=0.0):
    c, cam = s["c"], s["cam"]
    tot = 0.0
    for v, nu in enumerate(s["nus"]):
        for f, t in enumerate(s["times"]):
            img = oracle.polarized_image(c["a"], c["theta_o"], cam.alpha, cam.beta, s["N"], c["M"], [("thermal", p, None)], t, nu, c["L"],
                                         nmax=nmax, slab=slab)
            tot += float(np.sum(s["ds"][v, f] * img))
    return tot


def fd_gradient(oracle, s, nmax=-1, slab=0.0):
    p0 = s["p"]
    g = np.zeros_like(p0)
    for i in range(p0.shape[1]):
        for r in range(p0.shape[0]):
            h = 1e-7 * max(abs(p0[r, i]), 1.0)
            pp, pm = p0.copy(), p0.copy()
            pp[r, i] += h
            pm[r, i] -= h
            g[r, i] = (oracle_loss(oracle, s, pp, nmax, slab) - oracle_loss(oracle, s, pm, nmax, slab)) / (2 * h)
    return g


def compare(g, ref, tol):
    floor = 1e-4 * np.abs(ref).max()
    err = np.abs(g - ref) / (np.abs(ref) + floor)
    return err.max(), np.unravel_index(err.argmax(), err.shape)


@pytest.fixture(scope="module")
def fd(scene, oracle):
    oracle.set_threads(8)
    return fd_gradient(oracle, scene)


def test_fp64_adjoint_matches_finite_differences(scene, fd):
    s = scene
    g = ks.adjoint(s["cache"], ks.PolarizedSplats(s["p"]), s["times"], s["nus"], s["c"]["L"], s["ds"], precision=ks.KS_FP64)
    assert np.abs(fd).max() > 0
    err, where = compare(g, fd, 1e-5)
    print("fp64 adjoint vs FD: max rel err", err, "at (row, splat)", where)
    assert err < 1e-5, (err, where, g[where], fd[where])


def test_fp64_adjoint_is_deterministic_and_accumulates(scene):
    s = scene
    m = ks.PolarizedSplats(s["p"])
    g1 = ks.adjoint(s["cache"], m, s["times"], s["nus"], s["c"]["L"], s["ds"], precision=ks.KS_FP64)
    g2 = ks.adjoint(s["cache"], m, s["times"], s["nus"], s["c"]["L"], s["ds"], precision=ks.KS_FP64)
    assert np.array_equal(g1, g2)
    acc = np.asfortranarray(np.ones_like(g1))
    ks.adjoint(s["cache"], m, s["times"], s["nus"], s["c"]["L"], s["ds"], precision=ks.KS_FP64, dparams=acc)
    assert np.array_equal(acc, 1.0 + g1)


def test_chi2_gradient_matches_adjoint_of_its_seed(scene, oracle):
    s = scene
    c, cam = s["c"], s["cam"]
    m = ks.PolarizedSplats(s["p"])
    img = np.asarray(ks.render(s["cache"], m, s["times"], s["nus"], c["L"], precision=ks.KS_FP64))
    rng = np.random.Generator(np.random.PCG64(23))
    sigma = 0.05 * np.abs(img).max() * (1.0 + rng.uniform(0, 1, img.shape))
    data = img * (1 + 0.1 * rng.standard_normal(img.shape))
    mask = rng.uniform(0, 1, img.shape[:3]) > 0.2
    chi2, g, model = ks.chi2_gradient(s["cache"], m, s["times"], s["nus"], c["L"], data, sigma, mask=mask, precision=ks.KS_FP64,
                                      return_image=True)
    r = (img - data) / sigma * mask[..., None]
    assert np.allclose(model, img, rtol=1e-12, atol=1e-12 * np.abs(img).max())
    assert abs(chi2 - np.sum(r * r)) <= 1e-10 * np.sum(r * r)
    ga = ks.adjoint(s["cache"], m, s["times"], s["nus"], c["L"], 2 * r / sigma, precision=ks.KS_FP64)
    assert np.allclose(g, ga, rtol=1e-9, atol=1e-12 * np.abs(ga).max())
    # a scalar sigma
    chi2s, gs = ks.chi2_gradient(s["cache"], m, s["times"], s["nus"], c["L"], data, 0.1 * np.abs(img).max(), precision=ks.KS_FP64)
    rs = (img - data) / (0.1 * np.abs(img).max())
    assert abs(chi2s - np.sum(rs * rs)) <= 1e-10 * np.sum(rs * rs)


def test_truncated_adjoint_matches_finite_differences(oracle):
    # the half-orbit cutoff (winding_cutoff_kernel!): nmax = 0, a thin slab
    c = scenes.config2(res=8, N=48)
    rng = np.random.Generator(np.random.PCG64(24))
    p = scenes.thermal_params(rng, 2, c["a"], rlo=3.0, rhi=6.0)
    p[3:6] = np.log(rng.uniform(1.0, 2.0, (3, 2)))
    cam = ks.Camera((-8.0, 8.0), (-8.0, 8.0), 8)
    cache = ks.GeodesicCache(cam, 48)
    ks.regenerate(cache, c["a"], c["theta_o"])
    s = dict(c=c, p=p, cam=cam, times=np.array([0.0]), nus=np.array([230e9]), N=48)
    s["ds"] = rng.standard_normal((1, 1, cam.npix, 4))
    fdg = fd_gradient(oracle, s, nmax=0, slab=0.5)
    g = ks.adjoint(cache, ks.PolarizedSplats(p), s["times"], s["nus"], c["L"], s["ds"], nmax=0, slab=0.5, precision=ks.KS_FP64)
    err, where = compare(g, fdg, 1e-5)
    print("truncated fp64 adjoint vs FD:", err, where)
    assert err < 1e-5, (err, where)


def rel_l2(x, y):
    return float(np.linalg.norm(np.asarray(x) - np.asarray(y)) / max(np.linalg.norm(y), 1e-300))


def test_mixed_adjoint_matches_fp64(scene, fd):
    s = scene
    m = ks.PolarizedSplats(s["p"])
    g64 = ks.adjoint(s["cache"], m, s["times"], s["nus"], s["c"]["L"], s["ds"], precision=ks.KS_FP64)
    g32 = ks.adjoint(s["cache"], m, s["times"], s["nus"], s["c"]["L"], s["ds"], precision=ks.KS_MIXED)
    e64, e_fd = rel_l2(g32, g64), rel_l2(g32, fd)
    print("mixed adjoint: rel L2 vs fp64", e64, "vs FD", e_fd)
    assert e64 < 1e-3 and e_fd < 1e-3, (e64, e_fd)
    g32b = ks.adjoint(s["cache"], m, s["times"], s["nus"], s["c"]["L"], s["ds"], precision=ks.KS_MIXED)
    assert np.array_equal(g32, g32b)   # deterministic: fixed-order reductions, no atomics on the sums


@pytest.mark.parametrize("nus", [[86e9, 230e9, 345e9], [86e9, 230e9, 345e9, 690e9]])
def test_mixed_chi2_gradient_matches_fp64(nus):
    # three and four frequencies share a work unit of the mixed kernels (the configuration-2/3 layout)
    c = scenes.config2(res=12, N=96)
    rng = np.random.Generator(np.random.PCG64(25))
    p = scenes.thermal_params(rng, 6, c["a"], rlo=3.0, rhi=9.0)
    p[3:6] = np.log(rng.uniform(0.8, 2.0, (3, 6)))
    cam = ks.Camera((-12.0, 12.0), (-12.0, 12.0), 12)
    cache = ks.GeodesicCache(cam, 96)
    ks.regenerate(cache, c["a"], c["theta_o"])
    m = ks.PolarizedSplats(p)
    img = np.asarray(ks.render(cache, m, [0.0], nus, c["L"], precision=ks.KS_FP64))
    data = img * (1 + 0.05 * rng.standard_normal(img.shape))
    sigma = 0.01 * np.abs(img).max()
    chi64, g64 = ks.chi2_gradient(cache, m, [0.0], nus, c["L"], data, sigma, precision=ks.KS_FP64)
    chi32, g32 = ks.chi2_gradient(cache, m, [0.0], nus, c["L"], data, sigma, precision=ks.KS_MIXED)
    print("chi2", chi64, chi32, "grad rel L2", rel_l2(g32, g64))
    assert abs(chi32 - chi64) <= 1e-3 * chi64
    assert rel_l2(g32, g64) < 1e-3


def test_sample_adjoint_structured_matches_duals_and_fd(oracle):
    """sample_adjoint (transport.jl:221-245): the structured partials of the mixed path and the seven
    forward-mode duals of the FP64 path against each other (1e-10) and against central differences of
    the oracle's exact step (1e-6), over the linear, cubic and general branches of the step."""
    rng = np.random.Generator(np.random.PCG64(26))
    cam = ks.Camera((-1.0, 1.0), (-1.0, 1.0), 2)
    cache = ks.GeodesicCache(cam, 8)
    n = 60
    scale = np.concatenate([np.full(20, 1e-12), np.full(20, 1e-3), np.full(20, 1.0)])   # linear, cubic, general
    al = np.abs(rng.standard_normal((n, 4))) * scale[:, None]
    al[:, 0] += 2 * np.linalg.norm(al[:, 1:], axis=1)
    rh = rng.standard_normal((n, 3)) * scale[:, None] * 3
    j = np.abs(rng.standard_normal((n, 4)))
    coeffs = np.concatenate([j, al, rh], axis=1)
    Dl = rng.uniform(0.2, 3.0, n)
    w, R = rng.standard_normal((n, 4)), rng.standard_normal((n, 4))
    O0, E0, c0 = ks.sample_adjoint(cache, coeffs, Dl, w, R, method=0)
    O1, E1, c1 = ks.sample_adjoint(cache, coeffs, Dl, w, R, method=1)
    assert np.allclose(O0, O1, rtol=0, atol=1e-15) and np.allclose(E0, E1, rtol=0, atol=1e-15)
    den = np.abs(c1).max(axis=1, keepdims=True)
    assert np.max(np.abs(c0 - c1) / den) < 1e-10
    for i in range(n):
        def q(cf):
            O, E = oracle.transfer_step(cf[:4], cf[4:8], cf[8:11], Dl[i])
            return float(w[i] @ (O @ R[i] + E))
        for k in range(11):
            h = 1e-6 * max(abs(coeffs[i, k]), 0.1)
            cp, cm = coeffs[i].copy(), coeffs[i].copy()
            cp[k] += h
            cm[k] -= h
            fdv = (q(cp) - q(cm)) / (2 * h)
            assert abs(c0[i, k] - fdv) <= 1e-6 * den[i, 0] + 1e-6 * abs(fdv), (i, k, c0[i, k], fdv)


@pytest.mark.parametrize("prec,tol", [(ks.KS_FP64, 1e-6), (ks.KS_MIXED, 2e-3)])
def test_jvp_matches_finite_differences_and_adjoint(scene, oracle, prec, tol):
    """jvp! (gauss_newton.jl:91-118): J v of the image along random directions against central
    differences of the oracle image, and <dstokes, J v> = <J^T dstokes, v> against the adjoint."""
    s = scene
    c, cam = s["c"], s["cam"]
    m = ks.PolarizedSplats(s["p"])
    rng = np.random.Generator(np.random.PCG64(27))
    dirs = rng.standard_normal((3, 21, NS)) * np.maximum(np.abs(s["p"]), 0.1)[None]
    jv = ks.jvp(s["cache"], m, s["times"], s["nus"], c["L"], dirs, precision=prec)
    g = ks.adjoint(s["cache"], m, s["times"], s["nus"], c["L"], s["ds"], precision=ks.KS_FP64)
    for d in range(3):
        h = 1e-7
        fd = np.zeros_like(jv[d])
        for v, nu in enumerate(s["nus"]):
            for f, t in enumerate(s["times"]):
                ip = oracle.polarized_image(c["a"], c["theta_o"], cam.alpha, cam.beta, N, c["M"], [("thermal", s["p"] + h * dirs[d], None)], t,
                                            nu, c["L"])
                im = oracle.polarized_image(c["a"], c["theta_o"], cam.alpha, cam.beta, N, c["M"], [("thermal", s["p"] - h * dirs[d], None)], t,
                                            nu, c["L"])
                fd[v, f] = (ip - im) / (2 * h)
        e = rel_l2(jv[d], fd)
        dual = float(np.sum(s["ds"] * jv[d]))
        ref = float(np.sum(g * dirs[d]))
        print("jvp", prec, d, "rel L2 vs FD", e, "duality", dual, ref)
        assert e < tol, (d, e)
        assert abs(dual - ref) <= tol * abs(ref) + 1e-30, (d, dual, ref)
    # one direction (the one-partial pass the fit's Gauss-Newton curvature uses) equals the 8-wide pass:
    # the same arithmetic on Dual<S, 1> and Dual<S, 8>, which the compiler contracts into FMAs
    # differently, so they agree to the rounding of S (FP64 1e-9, FP32 duals 1e-5)
    jv1 = ks.jvp(s["cache"], m, s["times"], s["nus"], c["L"], dirs[:1], precision=prec)
    bound = 1e-9 if prec == ks.KS_FP64 else 1e-5
    assert rel_l2(jv1[0], jv[0]) < bound, rel_l2(jv1[0], jv[0])


@pytest.mark.parametrize("prec,tol", [(ks.KS_FP64, 1e-12), (ks.KS_MIXED, 1e-5)])
def test_normal_matrix(prec, tol):
    cam = ks.Camera((-1.0, 1.0), (-1.0, 1.0), 2)
    cache = ks.GeodesicCache(cam, 8)
    rng = np.random.Generator(np.random.PCG64(28))
    J = rng.standard_normal((1000, 77)) * np.exp(rng.uniform(-2, 2, 77))[None]
    A = ks.normal_matrix(cache, J, precision=prec)
    ref = J.T @ J
    assert np.max(np.abs(A - ref)) <= tol * np.abs(ref).max()


def test_spacetime_derivatives_match_oracle(scene, oracle):
    """The spacetime block (a, theta_o, ln L) of spacetime_valgrad (joint.jl:74-82), three-partial
    duals through the ray constants, anchors, march and transport, against the oracle's central
    differences (step 1e-5, the same discretised function: 1e-6)."""
    s = scene
    c, cam = s["c"], s["cam"]
    m = ks.PolarizedSplats(s["p"])
    h = 1e-5
    nu, t = s["nus"][:1], s["times"][:1]
    d, img = ks.spacetime_derivatives(s["cache"], m, t, nu, c["L"], precision=ks.KS_FP64, return_image=True)

    def orc(a, th, L):
        return oracle.polarized_image(a, th, cam.alpha, cam.beta, N, c["M"], [("thermal", s["p"], None)], t[0], nu[0], L)

    a, th, L = c["a"], c["theta_o"], c["L"]
    ref = [(orc(a + h, th, L) - orc(a - h, th, L)) / (2 * h), (orc(a, th + h, L) - orc(a, th - h, L)) / (2 * h),
           (orc(a, th, L * np.exp(h)) - orc(a, th, L * np.exp(-h))) / (2 * h)]
    errs = [rel_l2(d[q, 0, 0], ref[q]) for q in range(3)]
    print("spacetime derivatives rel L2 (a, theta_o, ln L):", errs)
    assert max(errs) < 1e-6, errs
    assert rel_l2(img[0, 0], orc(a, th, L)) < 1e-10
    # the context is unchanged
    again = np.asarray(ks.render(s["cache"], m, t, nu, L, precision=ks.KS_FP64))[0, 0]
    assert rel_l2(again, orc(a, th, L)) < 1e-10


def test_spacetime_derivatives_all_kinds():
    """The dual spacetime pass over thermal, power-law, kappa and knot splats, two frames and two
    frequencies, against central differences of the FP64 render (regenerated at a +- h, theta_o +- h;
    L e^(+-h)); its image equals the FP64 render (1e-12). A regenerate at a shifted spin or inclination
    can move a ray's anchor spacing (an integer of k) or carry a sample across the weight cutoff: the
    discretised function jumps there by ~1e-10 relative, which a central difference with one step turns
    into errors up to ~1e-4 at some pixels, while the duals keep those choices at the values. So each
    element is compared with the closest of the central differences at h = 1e-4, 1e-5, 1e-6: a jump
    spoils a step, not all three (rel L2 1e-6)."""
    a, tho = 0.94, np.deg2rad(163.0)
    rng = np.random.Generator(np.random.PCG64(41))
    pt = scenes.thermal_params(rng, 3, a)
    pp = scenes.powerlaw_params(rng, 3, a)
    pk = scenes.kappa_params(rng, 3, a)
    pn = scenes.thermal_params(rng, 2, a, rlo=3.0, rhi=7.0)
    pn[3:6] = np.log(rng.uniform(0.8, 2.0, (3, 2)))
    ktimes = np.array([-80.0, -30.0, 20.0, 60.0])
    model = ks.CompositeModel(ks.PolarizedSplats(pt), ks.PowerLawSplats(pp), ks.KappaSplats(pk),
                              ks.KnotSplats(pn, scenes.trajectory_knots(pn, a, ktimes), ktimes))
    cam = ks.Camera((-12.0, 12.0), (-12.0, 12.0), 12)
    cache = ks.GeodesicCache(cam, 96)
    L = ks.gravitational_radius(4e6)
    times, nus = [0.0, 20.0], [230e9, 690e9]
    ks.regenerate(cache, a, tho)
    d, img = ks.spacetime_derivatives(cache, model, times, nus, L, return_image=True)
    base = np.asarray(ks.render(cache, model, times, nus, L, precision=ks.KS_FP64))
    assert rel_l2(img, base) < 1e-12

    def rend(aa, th, LL):
        ks.regenerate(cache, aa, th)
        return np.asarray(ks.render(cache, model, times, nus, LL, precision=ks.KS_FP64))

    errs = []
    for q in range(3):
        fds = []
        for h in (1e-4, 1e-5, 1e-6):
            if q == 0:
                fds.append((rend(a + h, tho, L) - rend(a - h, tho, L)) / (2 * h))
            elif q == 1:
                fds.append((rend(a, tho + h, L) - rend(a, tho - h, L)) / (2 * h))
            else:
                fds.append((rend(a, tho, L * np.exp(h)) - rend(a, tho, L * np.exp(-h))) / (2 * h))
        fds = np.stack(fds)
        pick = np.argmin(np.abs(fds - d[q][None]), axis=0)
        best = np.take_along_axis(fds, pick[None], axis=0)[0]
        assert np.abs(best).max() > 0
        errs.append(rel_l2(d[q], best))
    ks.regenerate(cache, a, tho)
    print("spacetime derivatives, all kinds, rel L2 (a, theta_o, ln L):", errs)
    assert max(errs) < 1e-6, errs


def test_vis_chi2_gradient(scene, oracle):
    """The visibility chi^2 gradient of one frame (timeresolved_gradient!'s device path): the FP64
    call equals frame_chi2_seed followed by the adjoint seeded with its image seed (1e-9), a few
    components equal central differences of the oracle chi^2 (numpy DFT of oracle images, 1e-5),
    and the mixed call (3xTF32 DFT, FP32 transport) is within 1e-3 of FP64."""
    s = scene
    c, cam = s["c"], s["cam"]
    m = ks.PolarizedSplats(s["p"])
    t, nu = 0.0, 230e9
    rng = np.random.Generator(np.random.PCG64(29))
    nuv = 60
    rad = np.sqrt(rng.uniform(0, 1, nuv)) * 2e9
    ang = rng.uniform(0, 2 * np.pi, nuv)
    u, v = rad * np.cos(ang), rad * np.sin(ang)
    Dcm = 16.8e6 * 3.0857e18
    psize = (20.0 / (RES - 1)) * c["L"] / Dcm
    scale = psize ** 2 / 1e-23
    img = np.asarray(ks.render(s["cache"], m, [t], [nu], c["L"], precision=ks.KS_FP64))[0, 0]
    V = oracle.visibilities(img, RES, RES, u, v, None, psize, scale)
    vis = V * (1 + 0.1 * (rng.standard_normal(V.shape) + 1j * rng.standard_normal(V.shape)))
    sigma = 0.05 * np.abs(V).max() * np.ones((nuv, 4))
    chi64, g64 = ks.vis_chi2_gradient(s["cache"], m, t, nu, c["L"], u, v, vis, sigma, psize, scale, precision=ks.KS_FP64)
    chi_ref, seed = ks.frame_chi2_seed(s["cache"], img, u, v, vis, sigma, psize, scale, precision=ks.KS_FP64)
    g_ref = ks.adjoint(s["cache"], m, [t], [nu], c["L"], np.asarray(seed).reshape(1, 1, cam.npix, 4), precision=ks.KS_FP64)
    assert abs(chi64 - chi_ref) <= 1e-10 * chi_ref
    assert rel_l2(g64, g_ref) < 1e-9

    def ochi(p):
        im = oracle.polarized_image(c["a"], c["theta_o"], cam.alpha, cam.beta, N, c["M"], [("thermal", p, None)], t, nu, c["L"])
        return oracle.frame_chi2_seed(im, RES, RES, u, v, None, None, vis, sigma, psize, scale)[0]

    for (r, i) in [(12, 1), (13, 2), (0, 0), (17, 3), (20, 1)]:
        h = 1e-7 * max(abs(s["p"][r, i]), 1.0)
        pp, pm = s["p"].copy(), s["p"].copy()
        pp[r, i] += h
        pm[r, i] -= h
        fd = (ochi(pp) - ochi(pm)) / (2 * h)
        assert abs(g64[r, i] - fd) <= 1e-5 * max(abs(fd), 1e-4 * np.abs(g64).max()), (r, i, g64[r, i], fd)
    chi32, g32 = ks.vis_chi2_gradient(s["cache"], m, t, nu, c["L"], u, v, vis, sigma, psize, scale, precision=ks.KS_MIXED)
    print("vis chi2", chi64, chi32, "grad rel L2 mixed vs fp64", rel_l2(g32, g64))
    assert abs(chi32 - chi64) <= 1e-3 * chi64 and rel_l2(g32, g64) < 1e-3


def test_mixed_adjoint_large_splat_table():
    # 320 splats: the element kernel's per-unit gradient blocks live in global memory
    c = scenes.config2(res=12, N=64)
    rng = np.random.Generator(np.random.PCG64(30))
    p = scenes.thermal_params(rng, 320, c["a"], rlo=3.0, rhi=10.0)
    cam = ks.Camera((-12.0, 12.0), (-12.0, 12.0), 12)
    cache = ks.GeodesicCache(cam, 64)
    ks.regenerate(cache, c["a"], c["theta_o"])
    m = ks.PolarizedSplats(p)
    ds = rng.standard_normal((1, 1, cam.npix, 4))
    g64 = ks.adjoint(cache, m, [0.0], [230e9], c["L"], ds, precision=ks.KS_FP64)
    g32 = ks.adjoint(cache, m, [0.0], [230e9], c["L"], ds, precision=ks.KS_MIXED)
    print("320 splats: mixed vs fp64", rel_l2(g32, g64))
    assert np.abs(g64).max() > 0 and rel_l2(g32, g64) < 1e-3


def _crowded_scene():
    """480 wide splats (6 M) stacked on one spot (the FP64 plain adjoint stages at most 501): every
    sample near it passes every splat, so a block of the mixed kernels collects 384 x 256 pairs for a
    group of candidate words (past its pair list: the group is redone chunk by chunk) and 384 x 32 for
    one chunk (past it again: the chunk's list goes in two windows). The second block unit of the
    24 x 24 screen has dead warps."""
    c = scenes.config2(res=24, N=64)
    rng = np.random.Generator(np.random.PCG64(33))
    p = scenes.thermal_params(rng, 480, c["a"], rlo=5.5, rhi=6.5)
    p[0:3] = np.array([[6.0], [0.0], [0.5]]) + 0.2 * rng.standard_normal((3, 480))
    p[3:6] = np.log(6.0)
    p[12] = np.log(3e3)
    cam = ks.Camera((-12.0, 12.0), (-12.0, 12.0), 24)
    cache = ks.GeodesicCache(cam, 64)
    ks.regenerate(cache, c["a"], c["theta_o"])
    return c, p, cache


def test_crowded_pair_lists():
    """The mixed forward pass and chi^2 gradient on the crowded scene: the chunk-by-chunk and windowed
    pair lists give the FP64 plain results (image 1e-4, chi^2 1e-3, gradient 1e-3 rel L2)."""
    c, p, cache = _crowded_scene()
    m = ks.PolarizedSplats(p)
    nus = [230e9]
    img = np.asarray(ks.render(cache, m, [0.0], nus, c["L"], precision=ks.KS_FP64))
    mix = np.asarray(ks.render(cache, m, [0.0], nus, c["L"], precision=ks.KS_MIXED))
    assert np.abs(img).max() > 0
    e = rel_l2(mix, img)
    rng = np.random.Generator(np.random.PCG64(34))
    data = img * (1 + 0.05 * rng.standard_normal(img.shape))
    sigma = 0.01 * np.abs(img).max()
    chi64, g64 = ks.chi2_gradient(cache, m, [0.0], nus, c["L"], data, sigma, precision=ks.KS_FP64)
    chi32, g32 = ks.chi2_gradient(cache, m, [0.0], nus, c["L"], data, sigma, precision=ks.KS_MIXED)
    print("crowded: image rel L2", e, "chi2", chi64, chi32, "grad rel L2", rel_l2(g32, g64))
    assert e < 1e-4
    assert abs(chi32 - chi64) <= 1e-3 * chi64
    assert rel_l2(g32, g64) < 1e-3


def test_chi2_gradient_graph_replays_and_follows_parameters():
    """ks_chi2_gradient_graph_capture / ks_chi2_gradient_graph_launch: a mixed chi^2 + gradient of a
    device-resident thermal set against device-resident data, captured as a CUDA graph, replays to
    ks_chi2_gradient's chi^2 and gradient bit for bit. After an in-place change of the model's
    parameter buffer it replays to the new evaluation. A captured render survives the chi^2 capture,
    and a regenerate drops both graphs."""
    import torch
    c = scenes.config2(res=24, N=96)
    rng = np.random.Generator(np.random.PCG64(41))
    p = scenes.thermal_params(rng, 6, c["a"])
    cache = ks.GeodesicCache(c["camera"], c["N"])
    ks.regenerate(cache, c["a"], c["theta_o"])
    nus, times = [230e9, 345e9], [0.0]
    target = np.asarray(ks.render(cache, ks.PolarizedSplats(p * 1.02), times, nus, c["L"], precision=ks.KS_MIXED))
    sigma = 0.01 * float(np.abs(target[..., 0]).max())
    data = torch.tensor(target + sigma * rng.standard_normal(target.shape), device="cuda")
    model = ks.PolarizedSplats(torch.tensor(p, device="cuda"))
    rg = ks.capture_render(cache, model, times, nus, c["L"])

    def direct():
        buf = torch.zeros(21 * p.shape[1], dtype=torch.float64, device="cuda")
        chi2, _ = ks.chi2_gradient(cache, model, times, nus, c["L"], data, sigma, precision=ks.KS_MIXED, dparams=buf)
        return chi2, buf.cpu().numpy()

    g = ks.capture_chi2_gradient(cache, model, times, nus, c["L"], data, sigma)
    chi_ref, g_ref = direct()
    assert np.abs(g_ref).max() > 0
    chi2, dp = g.replay()
    assert float(chi2.item()) == chi_ref and np.array_equal(dp.cpu().numpy(), g_ref)
    model.sets()[0].params[:, 12] += np.log(1.2)   # the log densities, in place
    chi_ref2, g_ref2 = direct()
    assert chi_ref2 != chi_ref
    chi2, dp = g.replay()
    assert float(chi2.item()) == chi_ref2 and np.array_equal(dp.cpu().numpy(), g_ref2)
    rg.replay()   # the render graph is still there
    ks.regenerate(cache, c["a"], c["theta_o"])
    with pytest.raises(ValueError, match="no captured chi"):
        g.replay()
    with pytest.raises(ValueError, match="no captured graph"):
        rg.replay()
    cache.close()
