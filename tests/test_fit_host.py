"""Host logic of kerrsplat_b200.fit (CPU only): LSQR against the dense damped least-squares solution,
the residual layout's round trip, and the gain factors."""
import numpy as np

from kerrsplat_b200 import fit


def test_lsqr_matches_dense_damped_least_squares():
    rng = np.random.default_rng(0)
    m, n = 60, 25
    # a conditioned-but-not-trivial operator: singular values over three decades
    U, _ = np.linalg.qr(rng.standard_normal((m, n)))
    V, _ = np.linalg.qr(rng.standard_normal((n, n)))
    A = U @ np.diag(np.logspace(0, -3, n)) @ V.T
    r = rng.standard_normal(m)
    for damp in (0.0, 1e-2, 0.3):
        x, k, rel = fit.lsqr(lambda v: A @ v, lambda u: A.T @ u, r, damp=damp, iterations=400, atol=1e-12)
        ref = np.linalg.solve(A.T @ A + damp ** 2 * np.eye(n), -A.T @ r)
        assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < 1e-8, (damp, k, rel)
        assert rel <= 1e-12 or k == 400
    # the relative normal-equation residual decreases and stops the iterations at atol
    x, k, rel = fit.lsqr(lambda v: A @ v, lambda u: A.T @ u, r, damp=0.1, iterations=200, atol=1e-4)
    assert rel <= 1e-4 and k < 200
    # a zero right-hand side is a zero step
    x, k, rel = fit.lsqr(lambda v: A @ v, lambda u: A.T @ u, np.zeros(m))
    assert k == 0 and np.all(x == 0)


def test_residual_layout_and_gains():
    rng = np.random.default_rng(1)
    z = rng.standard_normal((7, 4)) + 1j * rng.standard_normal((7, 4))
    f = fit._flat(z)
    assert f.shape == (56,)
    assert np.array_equal(f[:8], [z[0, 0].real, z[0, 0].imag, z[0, 1].real, z[0, 1].imag, z[0, 2].real, z[0, 2].imag, z[0, 3].real,
                                  z[0, 3].imag])
    assert np.array_equal(fit._unflat(f, 7), z)
    gains = np.array([[0.1, -0.2, 0.05], [0.3, 0.0, -1.0]])
    g = fit.FrameScans.gain_factors(gains, [0, 1], [2, 0])
    want = [np.exp(0.1 + 0.3j) * np.conj(np.exp(0.05 - 1.0j)), np.exp(-0.2) * np.conj(np.exp(0.1 + 0.3j))]
    assert np.allclose(g, want, rtol=1e-15)
    fs = fit.FrameScans(rng.standard_normal(7), rng.standard_normal(7), z, 0.5)
    assert fs.nres == 56 and fs.sigma.shape == (7, 4) and np.all(fs.g == 1)
    b = fit.BandScans({10.0: fs, 0.0: fs}, 230e9, 1e-11, 1.0)
    assert list(b.times) == [0.0, 10.0] and b.nres == 112 and fit.residual_length([b, b]) == 224


def test_adam_steps_toward_a_quadratic_minimum():
    target = np.array([[1.0, -2.0], [0.5, 3.0]])
    valgrad = lambda p: (float(np.sum((p - target) ** 2)), 2 * (p - target))
    p, hist = fit.fit(valgrad, np.zeros((2, 2)), iterations=2000, lr=0.05)
    assert hist[-1] < 1e-6 * hist[0] and np.allclose(p, target, atol=1e-3)
