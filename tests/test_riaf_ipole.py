"""Pin of the frames and the composed polarized transport against ipole (CPU only).

The reference compares its full-Stokes images of ipole's example RIAF (test/riaf_model.jl: thick
disk, toroidal field, Keplerian rotation with the plunge inside the ISCO, thermal synchrotron with
Pandya emissivities) with ipole's own images (validation/ipole_riaf/, extracted into
tests/golden/ipole_riaf.npz by tests/golden/make_golden.py). This restates that comparison on the
oracle: the same 100 x 100 camera (ipole's pixel centres), a = 0.9375, theta_o = 85 deg,
Recurrence(64) with N = 2000 samples per ray, 230 GHz (Faraday depths up to 9 rad) and 2 THz
(intrinsic polarization only), and the reference's own gate (test/test_polarized.jl:156-178):
per-Stokes pixel-norm residual < 0.03, totals within 1%, median EVPA difference < 0.01 rad over
pixels brighter than 1% of the peak, and median linear-polarization fraction within 0.005.

The screen angle chi, the ZAMO axes, the boost and the Walker-Penrose transport enter Q and U: a
mirrored chi (planted in the oracle) fails the same gate.
"""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PC, JY = 3.085678e18, 1e-23
A, THETA_O, MBH, DIST = 0.9375, np.deg2rad(85.0), 4.3e6, 8.3e3 * PC


def gravitational_radius(msun):
    return 6.6742e-8 * msun * 1.989e33 / 2.99792458e10 ** 2


def riaf_camera(res=100):
    """ipole's pixel centres (x offset (i + 0.49)/nx - 0.5, y offset (j + 0.5)/ny - 0.5, in units
    of the field of view), pixel i + j res (test/test_polarized.jl:140-151)."""
    L = gravitational_radius(MBH)
    fov = 200e-6 / 206264.806247 * DIST / L
    xs = ((np.arange(res) + 0.49) / res - 0.5) * fov
    ys = ((np.arange(res) + 0.5) / res - 0.5) * fov
    i, j = np.meshgrid(np.arange(res), np.arange(res), indexing="ij")
    alpha = xs[i].ravel(order="F")
    beta = ys[j].ravel(order="F")
    scale = (fov / res * L / DIST) ** 2 / JY
    return alpha, beta, L, scale


def ipole_reference(tag):
    z = np.load(os.path.join(GOLDEN, "ipole_riaf.npz"))
    return np.stack([z[f"{tag}_{s}"].ravel(order="F") for s in "IQUV"], axis=1)   # [i, j] -> pixel i + j res


def gate(ours, ref, scale):
    """The reference's comparison (test/test_polarized.jl:162-173): returns residuals, total ratios,
    median EVPA difference and the two median polarization fractions."""
    res = np.array([np.linalg.norm(ours[:, k] - ref[:, k]) / np.linalg.norm(ref[:, k]) for k in range(4)])
    tot = ours.sum(axis=0) * scale / (ref.sum(axis=0) * scale)
    w = ref[:, 0] > 0.01 * ref[:, 0].max()
    chi_o = 0.5 * np.arctan2(ours[:, 2], ours[:, 1])
    chi_r = 0.5 * np.arctan2(ref[:, 2], ref[:, 1])
    d = chi_o - chi_r
    d = d - np.pi * np.round(d / np.pi)                 # rem(., pi, RoundNearest)
    dchi = np.median(np.abs(d[w]))
    lp = np.median(np.hypot(ours[w, 1], ours[w, 2]) / ours[w, 0])
    lpr = np.median(np.hypot(ref[w, 1], ref[w, 2]) / ref[w, 0])
    return res, tot, dchi, lp, lpr


def test_pandya_emissivities_vs_symphony(oracle):
    """thermal_synchrotron_pandya against the symphony table's jI/jQ/jV_pandya columns at 1e-12
    (test/test_coefficients.jl:50-53)."""
    import csv
    with open(os.path.join(GOLDEN, "symphony_thermal_table.csv")) as f:
        rows = list(csv.DictReader(f))
    t = {k: np.array([float(r[k]) for r in rows]) for k in rows[0]}
    out = oracle.thermal(t["ne"], t["Thetae"], t["B"], t["nu"], t["theta"], pandya=True)
    for k, name in ((0, "jI_pandya"), (1, "jQ_pandya"), (2, "jV_pandya")):
        err = np.abs(out[:, k] - t[name]) / np.maximum(np.abs(t[name]), 1e-280)
        assert err.max() < 1e-12, (name, err.max())
    # the absorptivities stay Kirchhoff's law of the emissivities in use
    bnu = out[:, 0] / out[:, 3]
    assert np.allclose(out[:, 4] * bnu, out[:, 1], rtol=1e-12)


@pytest.mark.parametrize("tag,nu", [("fine", 230e9), ("2thz", 2e12)])
def test_riaf_full_stokes_matches_ipole(oracle, tag, nu):
    alpha, beta, L, scale = riaf_camera()
    ours = oracle.riaf_image(A, THETA_O, alpha, beta, 2000, 64, nu, L, pandya=True)
    ref = ipole_reference(tag)
    res, tot, dchi, lp, lpr = gate(ours, ref, scale)
    msg = f"{tag}: residuals {res}, totals {tot}, dchi {dchi:.2e}, lp {lp:.4f} vs {lpr:.4f}"
    print(msg)
    assert np.all(res < 0.03), msg
    assert np.all(np.abs(tot - 1) < 0.01), msg
    assert dchi < 0.01, msg
    assert abs(lp - lpr) < 0.005, msg


def test_riaf_gate_rejects_a_mirrored_screen_angle(oracle):
    """A sign error in chi (planted in the oracle) leaves I and the polarized fraction but turns the
    EVPA: the gate must fail it. Every 7th pixel at 2 THz, where chi alone sets Q and U."""
    alpha, beta, L, scale = riaf_camera()
    sel = slice(0, None, 7)
    ref = ipole_reference("2thz")[sel]
    good = oracle.riaf_image(A, THETA_O, alpha[sel], beta[sel], 2000, 64, 2e12, L)
    bad = oracle.riaf_image(A, THETA_O, alpha[sel], beta[sel], 2000, 64, 2e12, L, mirror_chi=True)
    res_g, _, dchi_g, _, _ = gate(good, ref, scale)
    res_b, _, dchi_b, _, _ = gate(bad, ref, scale)
    assert np.all(res_g < 0.03) and dchi_g < 0.01
    assert res_b[0] < 0.03                      # I does not see chi
    assert res_b[2] > 0.03 or dchi_b > 0.01     # U (and the EVPA) do
    assert dchi_b > 0.01
