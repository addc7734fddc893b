"""Pins of the CPU oracle (CPU only): against the reference's committed golden data (symphony
coefficient tables) and against the mpmath restatements of the reference's BigFloat references
(tests/golden/make_golden.py). The tolerances are the reference's own (test_coefficients.jl:29-70,
test_recurrence.jl:6-15, runtests.jl:46, test_transfer_step.jl)."""
import csv
import json
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def table(name):
    with open(os.path.join(GOLDEN, name)) as f:
        rows = list(csv.DictReader(f))
    return {k: np.array([float(r[k]) for r in rows]) for k in rows[0]}


def relerr(a, b):
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-280)


def test_thermal_coefficients_vs_symphony(oracle):
    t = table("symphony_thermal_table.csv")
    out = oracle.thermal(t["ne"], t["Thetae"], t["B"], t["nu"], t["theta"])
    for k, name in enumerate(["jI", "jQ", "jV", "aI", "aQ", "aV", "rhoQ", "rhoV"]):
        assert relerr(out[:, k], t[name]).max() < 1e-12, name
    dex = oracle.thermal(t["ne"], t["Thetae"], t["B"], t["nu"], t["theta"], dexter_rhoV=True)
    assert relerr(dex[:, 7], t["rhoV_dexter"]).max() < 1e-12


def test_powerlaw_coefficients_vs_symphony(oracle):
    t = table("symphony_powerlaw_table.csv")
    out = oracle.powerlaw(t["ne"], t["p"], t["gamma_min"], t["gamma_max"], t["B"], t["nu"], t["theta"])
    for k, name in enumerate(["jI", "jQ", "jV", "aI", "aQ", "aV"]):
        assert relerr(out[:, k], t[name]).max() < 1e-12, name


def test_powerlaw_rotativities_vs_symphony(oracle):
    """Jones & O'Dell closed forms vs symphony's numerical susceptibilities: sign everywhere, 5% in
    rho_V and 35% in rho_Q inside nu > 3 gamma_min^2 nu_B (test_coefficients.jl:131-159)."""
    t = table("symphony_powerlaw_rho_table.csv")
    EE, ME, CL = 4.80320680e-10, 9.1093826e-28, 2.99792458e10
    valid = t["nu"] > 3 * t["gamma_min"] ** 2 * EE * t["B"] * np.sin(t["theta"]) / (2 * np.pi * ME * CL)
    out = oracle.powerlaw(t["ne"], t["p"], t["gamma_min"], t["gamma_max"], t["B"], t["nu"], t["theta"])
    rq, rv = out[valid, 6], out[valid, 7]
    assert np.all(np.sign(rq) == np.sign(t["rhoQ"][valid])) and np.all(np.sign(rv) == np.sign(t["rhoV"][valid]))
    assert np.max(np.abs(rv / t["rhoV"][valid] - 1)) < 0.05
    assert np.max(np.abs(rq / t["rhoQ"][valid] - 1)) < 0.35


def test_kappa_coefficients_vs_symphony(oracle):
    import mpmath
    t = table("symphony_kappa_table.csv")
    hyp = np.array([float(mpmath.hyp2f1(k - 1 / 3, k + 1, k + 2 / 3, -k * w)) for k, w in zip(t["kappa"], t["w"])])
    out = oracle.kappa(t["ne"], t["kappa"], t["w"], t["B"], t["nu"], t["theta"], hyp)
    for k, name in [(0, "jI"), (1, "jQ"), (3, "aI"), (4, "aQ"), (5, "aV"), (6, "rhoQ"), (7, "rhoV")]:
        sel = np.ones_like(t["nu"], dtype=bool) if name != "rhoQ" else t["kappa"] != 5.0
        assert relerr(out[sel, k], t[name][sel]).max() < 1e-10, name
    nz = t["jV"] != 0
    assert relerr(out[nz, 2], t["jV"][nz]).max() < 1e-10


def test_special_functions(oracle):
    d = json.load(open(os.path.join(GOLDEN, "special_pins.json")))
    x = np.array([b["x"] for b in d["bessel"]])
    k0, k1 = oracle.besselk01(x)
    assert relerr(k0, np.array([b["k0"] for b in d["bessel"]])).max() < 1e-14
    assert relerr(k1, np.array([b["k1"] for b in d["bessel"]])).max() < 1e-14
    phi = np.array([e["phi"] for e in d["ellipf"]]); m = np.array([e["m"] for e in d["ellipf"]])
    F = oracle.ellipf(phi, m)
    assert relerr(F, np.array([e["F"] for e in d["ellipf"]])).max() < 1e-13
    u = np.array([e["u"] for e in d["jacobi"]]); m = np.array([e["m"] for e in d["jacobi"]])
    sn, cn, dn = oracle.jacobi_state(u, m)
    for got, key in ((sn, "sn"), (cn, "cn"), (dn, "dn")):
        assert np.max(np.abs(got - np.array([e[key] for e in d["jacobi"]]))) < 1e-12, key


def test_transfer_step_vs_matrix_exponential(oracle):
    """The closed-form step vs exp of the augmented matrix in 40-digit arithmetic, across the
    regimes the closed forms switch between (test_transfer_step.jl:21-80; tolerance 1e-13 there
    relative to the operator norms)."""
    cases = json.load(open(os.path.join(GOLDEN, "step_pins.json")))
    worst_O = worst_E = 0.0
    for c in cases:
        O, E = oracle.transfer_step(c["j"], c["alpha"], c["rho"], c["D"])
        Oref, Eref = np.array(c["O"]), np.array(c["E"])
        worst_O = max(worst_O, np.linalg.norm(O - Oref) / max(np.linalg.norm(Oref), 1e-300))
        worst_E = max(worst_E, np.linalg.norm(E - Eref) / max(np.linalg.norm(Eref), 1e-300))
    assert worst_O < 1e-11 and worst_E < 1e-11, (worst_O, worst_E)


def test_step_physics(oracle):
    """Kirchhoff equilibrium, Faraday rotation as a rotation, the semigroup property."""
    # equilibrium: j = alpha_I * S_eq with S_eq = (1, 0, 0, 0) unpolarized and no polarized terms
    O, E = oracle.transfer_step([2.0, 0, 0, 0], [2.0, 0, 0, 0], [0, 0, 0], 3.0)
    S = O @ np.array([1.0, 0, 0, 0]) + E
    assert np.allclose(S, [1, 0, 0, 0], atol=1e-13)
    # pure Faraday rotation (rho_V) rotates (Q, U) by 2 * rho_V * D... and keeps I, V and |P|
    O, E = oracle.transfer_step([0, 0, 0, 0], [0, 0, 0, 0], [0, 0, 0.7], 1.3)
    S = O @ np.array([1.0, 0.6, 0.0, 0.2])
    assert abs(S[0] - 1) < 1e-14 and abs(S[3] - 0.2) < 1e-14 and abs(np.hypot(S[1], S[2]) - 0.6) < 1e-14
    # semigroup: two half steps = one step
    j, a, r = [1.0, 0.3, -0.2, 0.1], [0.8, 0.2, 0.1, -0.05], [0.4, -0.3, 1.1]
    O1, E1 = oracle.transfer_step(j, a, r, 0.35)
    O2, E2 = oracle.transfer_step(j, a, r, 0.7)
    assert np.allclose(O1 @ O1, O2, atol=1e-13) and np.allclose(O1 @ E1 + E1, E2, atol=1e-13)


def load_pins(name):
    path = os.path.join(GOLDEN, name)
    if not os.path.exists(path):
        pytest.skip(f"{name} not generated")
    return json.load(open(path))


def test_recurrence_r_theta_vs_highprec(oracle):
    """Gate 2: r and theta of the recurrence march vs the 40-digit closed forms at the pinned
    samples, 1e-10 (relative in r) or the root-limited accuracy near the critical curve
    (test_recurrence.jl:6-15)."""
    pins = load_pins("geodesic_pins.json")
    worst = 0.0
    for p in pins:
        s = oracle.march_samples(p["a"], p["theta_o"], np.array([p["alpha"]]), np.array([p["beta"]]), p["N"], 64)
        rc = oracle.ray_constants(p["a"], p["theta_o"], np.array([p["alpha"]]), np.array([p["beta"]]))[0]
        tol = 1e-10 if 1 - rc[3] > 1e-4 else 1e-7
        for q in p["samples"]:
            k = q["k"] - 1
            er = abs(s["r"][0, k] - q["r"]) / max(q["r"], 1.0)
            et = abs(s["theta"][0, k] - q["theta"])
            worst = max(worst, er if tol == 1e-10 else 0.0)
            assert er < tol and et < 1e-10, (p["alpha"], p["beta"], q["k"], er, et)
    assert worst < 1e-10


def test_quadrature_increments_vs_highprec(oracle):
    """Gate 3: increments of t~ and phi from the first sample inside 50 M vs 16-point
    Gauss-Legendre of the rates in 40 digits; tol_hp_t = 2e-8, tol_hp_phi = 2e-9 (runtests.jl:46)."""
    pins = load_pins("geodesic_pins.json")
    for p in pins:
        if len(p["increments"]) < 2:
            continue
        s = oracle.march_samples(p["a"], p["theta_o"], np.array([p["alpha"]]), np.array([p["beta"]]), p["N"], 64)
        k1 = p["increments"][0]["k"] - 1
        for q in p["increments"][1:]:
            k = q["k"] - 1
            dt = s["t"][0, k] - s["t"][0, k1]
            dp = s["phi"][0, k] - s["phi"][0, k1]
            assert abs(dt - q["dt"]) < 2e-8 and abs(dp - q["dphi"]) < 2e-9, (p["alpha"], p["beta"], q["k"], dt - q["dt"], dp - q["dphi"])


def test_anchor_values_vs_highprec(oracle):
    """Absolute regularized t~ and phi of the anchor evaluator vs adaptive 40-digit quadrature of
    the rates from the observer (the regularization drops r_obs + 2 ln r_obs)."""
    pins = load_pins("anchor_pins.json")
    for p in pins:
        t, ph, ok = oracle.anchor_values(p["a"], p["theta_o"], np.array([p["alpha"]]), np.array([p["beta"]]), p["N"])
        for v in p["values"]:
            k = v["k"] - 1
            assert abs(t[0, k] - v["t"]) < 1e-9 * max(1.0, abs(v["t"])), (p["alpha"], p["beta"], v["k"], t[0, k], v["t"])
            assert abs(ph[0, k] - v["phi"]) < 1e-9, (p["alpha"], p["beta"], v["k"], ph[0, k], v["phi"])


def test_recurrence_matches_direct_anchors(oracle):
    """The recurrence + Simpson quadrature stays within 1e-8 of the anchor evaluator at every
    sample of a 32x32 config-1 screen (the reference's per-ray anchor residuals are of this order)."""
    from kerrsplat_b200 import scenes
    c = scenes.config1(res=16, N=256)
    cam = c["camera"]
    s = oracle.march_samples(c["a"], c["theta_o"], cam.alpha, cam.beta, c["N"], 64)
    assert np.max(s["resid_t"]) < 1e-7 and np.max(s["resid_phi"]) < 1e-8
