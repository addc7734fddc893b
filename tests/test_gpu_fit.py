"""The fit-loop products on the GPU (kerrsplat_b200.fit): J v and J^T w in residual space against each
other (<w, J v> = <J^T w, v>) and against central differences of the residuals, the time-resolved
chi^2 gradient against 2 J^T r, LSQR against the dense damped solution on a few free parameters,
and a Levenberg-Marquardt polish and an Adam fit that lower chi^2. A small scene: five thermal
splats on a 12 x 12 screen, two frames, 24 baselines per frame with gains."""
import numpy as np
import pytest

import kerrsplat_b200 as ks
from kerrsplat_b200 import fit, scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def problem():
    c = scenes.config2(res=12, N=64)
    rng = np.random.Generator(np.random.PCG64(71))
    p = scenes.thermal_params(rng, 5, c["a"], rlo=3.0, rhi=8.0)
    p[3:6] = np.log(rng.uniform(1.0, 2.5, (3, 5)))
    cam = ks.Camera((-10.0, 10.0), (-10.0, 10.0), 12)
    cache = ks.GeodesicCache(cam, 64)
    ks.regenerate(cache, c["a"], c["theta_o"])
    L = c["L"]
    D = 8.3e3 * 3.085678e18
    psize = (20.0 / 11) * L / D
    scale = psize ** 2 / 1e-23
    nu = 230e9
    truth = p + 0.03 * np.maximum(np.abs(p), 0.1) * rng.standard_normal(p.shape)
    frames = {}
    imgs = np.asarray(ks.render(cache, ks.PolarizedSplats(truth), [0.0, 20.0], [nu], L, precision=ks.KS_FP64))[0]
    for f, t in enumerate((0.0, 20.0)):
        nuv = 24
        rad = 2e10 * np.sqrt(rng.uniform(0, 1, nuv))
        ang = rng.uniform(0, 2 * np.pi, nuv)
        u, v = rad * np.cos(ang), rad * np.sin(ang)
        V = ks.visibilities(cache, imgs[f], u, v, psize, scale, precision=ks.KS_FP64)
        gains = np.array([rng.normal(0, 0.05, 4), rng.uniform(-0.3, 0.3, 4)])
        s1, s2 = rng.integers(0, 4, nuv), rng.integers(0, 4, nuv)
        g = fit.FrameScans.gain_factors(gains, s1, s2)
        sigma = 0.02 * np.sqrt(np.mean(np.abs(V) ** 2, axis=0))[None, :] * np.ones((nuv, 1))
        data = g[:, None] * V + sigma * (rng.standard_normal((nuv, 4)) + 1j * rng.standard_normal((nuv, 4)))
        frames[t] = fit.FrameScans(u, v, data, sigma, g=g)
    band = fit.BandScans(frames, nu, psize, scale)
    yield dict(cache=cache, p=p, L=L, band=band, rng=rng)
    cache.close()


def test_jvp_jtvp_adjoint_identity_and_fd(problem):
    s = problem
    rng = np.random.default_rng(5)
    v = rng.standard_normal(s["p"].shape) * np.maximum(np.abs(s["p"]), 0.1) * 1e-2
    w = rng.standard_normal(s["band"].nres)
    for prec, tol in ((ks.KS_FP64, 1e-10), (ks.KS_MIXED, 1e-4)):
        Jv = fit.jvp(s["cache"], s["p"], s["band"], s["L"], v, precision=prec)
        Jtw = fit.jtvp(s["cache"], s["p"], s["band"], s["L"], w, precision=prec)
        lhs, rhs = float(w @ Jv), float(np.sum(Jtw * v))
        print("adjoint identity", prec, lhs, rhs)
        assert abs(lhs - rhs) < tol * max(abs(lhs), abs(rhs))
    # J v against central differences of the residuals (FP64)
    h = 1e-4
    rp, _ = fit.residuals(s["cache"], s["p"] + h * v, s["band"], s["L"], precision=ks.KS_FP64)
    rm, _ = fit.residuals(s["cache"], s["p"] - h * v, s["band"], s["L"], precision=ks.KS_FP64)
    fd = (rp - rm) / (2 * h)
    Jv = fit.jvp(s["cache"], s["p"], s["band"], s["L"], v, precision=ks.KS_FP64)
    err = np.linalg.norm(Jv - fd) / np.linalg.norm(fd)
    print("J v vs central differences", err)
    assert err < 1e-5


def test_timeresolved_gradient_is_twice_jt_r(problem):
    s = problem
    for prec, tol in ((ks.KS_FP64, 1e-9), (ks.KS_MIXED, 1e-3)):
        chi, g = fit.timeresolved_gradient(s["cache"], s["p"], s["band"], s["L"], precision=prec)
        r, chi_r = fit.residuals(s["cache"], s["p"], s["band"], s["L"], precision=prec)
        jt = fit.jtvp(s["cache"], s["p"], s["band"], s["L"], r, precision=prec)
        e = np.linalg.norm(g - 2 * jt) / np.linalg.norm(g)
        print("time-resolved gradient", prec, chi, chi_r, e)
        assert abs(chi - chi_r) < tol * chi
        assert e < tol


def test_lsqr_step_matches_dense_solution(problem):
    s = problem
    p, band, L = s["p"], s["band"], s["L"]
    free = np.zeros_like(p)
    idx = [(12, 0), (13, 1), (14, 2), (0, 3), (20, 4), (17, 0)]
    for r_, c_ in idx:
        free[r_, c_] = 1.0
    S = free * 0.1
    r, _ = fit.residuals(s["cache"], p, band, L, precision=ks.KS_FP64)
    x, k, rel = fit.lsqr_step(s["cache"], p, band, L, r, S, damp=0.05, iterations=30, atol=1e-12, precision=ks.KS_FP64)
    # the dense Jacobian of the free columns, scaled
    E = np.zeros((len(idx),) + p.shape)
    for q, (r_, c_) in enumerate(idx):
        E[q, r_, c_] = S[r_, c_]
    J = fit.jvp(s["cache"], p, band, L, E, precision=ks.KS_FP64).T       # (m, nfree)
    ref = np.linalg.solve(J.T @ J + 0.05 ** 2 * np.eye(len(idx)), -J.T @ r)
    got = np.array([x[r_, c_] for r_, c_ in idx])
    print("LSQR", k, rel, got, ref)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-6
    assert np.all(x[free == 0] == 0)


def test_polish_and_adam_lower_chi2(problem):
    s = problem
    p, band, L = s["p"], s["band"], s["L"]
    free = np.zeros_like(p)
    free[12:15] = 1.0          # densities, temperatures, field strengths
    p1, hist = fit.polish_timeresolved(s["cache"], p, band, L, iterations=3, solve_iterations=10, probes=2, free=free,
                                       rng=np.random.default_rng(2))
    print("polish chi2", hist)
    assert hist[-1] < 0.5 * hist[0]
    assert np.all(p1[free == 0] == p[free == 0])
    # the image-domain fit (fit!'s dual value-and-gradient, Adam on the host)
    cache = s["cache"]
    truth = p.copy()
    truth[12] += 0.2
    data = np.asarray(ks.render(cache, ks.PolarizedSplats(truth), [0.0], [230e9], L, precision=ks.KS_FP64))
    sigma = 0.01 * np.abs(data[..., 0]).max()
    vg = lambda q: fit.dual_valgrad(cache, q, [0.0], [230e9], L, data, sigma)
    sc = np.zeros_like(p)
    sc[12] = 1.0               # only the log-densities move
    q, hist2 = fit.fit(vg, p, iterations=40, lr=0.02, scale=sc)
    print("adam chi2", hist2[0], hist2[-1])
    assert hist2[-1] < 0.2 * hist2[0]


def test_graph_valgrad_matches_dual_valgrad(problem):
    """fit.GraphValgrad (the evaluation captured once, replayed per call) against fit.dual_valgrad with
    the mixed path: the same chi^2 and gradient bit for bit at the starting parameters. Ten Adam steps
    on each follow the same trajectory."""
    s = problem
    p, L, cache = s["p"], s["L"], s["cache"]
    truth = p.copy()
    truth[12] += 0.2
    data = np.asarray(ks.render(cache, ks.PolarizedSplats(truth), [0.0], [230e9], L, precision=ks.KS_FP64))
    sigma = 0.01 * np.abs(data[..., 0]).max()
    direct = lambda q: fit.dual_valgrad(cache, q, [0.0], [230e9], L, data, sigma, precision=ks.KS_MIXED)
    graph = fit.GraphValgrad(cache, p, [0.0], [230e9], L, data, sigma)
    c0, g0 = direct(p)
    c1, g1 = graph(p)
    assert c1 == c0 and g1.shape == g0.shape and np.array_equal(g1, g0)
    sc = np.zeros_like(p)
    sc[12] = 1.0
    qa, ha = fit.fit(direct, p, iterations=10, lr=0.02, scale=sc)
    qb, hb = fit.fit(graph, p, iterations=10, lr=0.02, scale=sc)
    assert np.array_equal(np.asarray(ha), np.asarray(hb)) and np.array_equal(qa, qb)
    assert hb[-1] < hb[0]
    graph.close()
