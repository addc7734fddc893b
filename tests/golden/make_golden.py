"""Generate the golden fixtures under tests/golden/ (run once, here; the outputs are committed).

Two kinds of fixtures:

1. Extracts of the reference's own committed golden data. Needs the reference checkout, named by
   the REFERENCE_ROOT environment variable or the `--reference <dir>` argument (no default):
   * validation/symphony/*.csv, the symphony-generated coefficient tables that
     test/test_coefficients.jl compares against at 1e-12: every 4th row, the columns the tests use;
   * validation/ipole_riaf/riaf_{fine,2thz}_{I,Q,U,V}.csv, ipole's full-Stokes images of its
     example RIAF at 230 GHz and 2 THz (100 x 100, row = x index, column = y index), which
     test/test_polarized.jl:156-178 compares KerrSplat's images against: all eight arrays as float64
     in one compressed file, ipole_riaf.npz (keys "fine_I" ... "2thz_V");
   * test/data/synth_eht2017{,_noiseless}.uvfits, their parses by ehtim (*_ehtim.csv) and the source
     image synth_eht2017_image.fits, which test/test_uvfits.jl pins the uvfits reader, the FITS
     image reader and the sky conventions of the transform against: copied unchanged into
     tests/golden/uvfits/.
2. High-precision references restated in mpmath (the reference's own BigFloat references are
   Julia, test/highprec_reference.jl and test/test_transfer_step.jl):
   * r(tau), theta(tau) from the closed forms with Newton-polished roots (highprec_reference.jl:22-156);
   * increments of t~ and phi by 16-point Gauss-Legendre quadrature of the Mino-time rates
     (highprec_reference.jl:183-221);
   * absolute t~ and phi (the anchors) by adaptive quadrature of the rates from the observer, t~
     regularized by dropping r_obs + 2 ln r_obs (docs/notes/2026-09-03_phase3_slowlight.md:6-8);
   * the exact transfer step by the matrix exponential of the augmented 8x8 matrix
     [[-K, I], [0, 0]] Delta (Van Loan 1978), which holds exp(-K Delta) and int_0^Delta exp(-K u) du;
   * K0, K1, F(phi|m), and (sn, cn, dn)(u|m).
The rays come from the oracle's own Float64 roots (as the reference's BigFloat reference starts from
Krang's), so the oracle library must be built (make -C oracle).
"""
import csv
import json
import os
import sys

import mpmath as mp
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle  # noqa: E402

REFERENCE_ROOT = os.environ.get("REFERENCE_ROOT")


def reference_root():
    if not REFERENCE_ROOT:
        raise SystemExit("name the reference checkout: REFERENCE_ROOT=<dir> or --reference <dir>")
    return REFERENCE_ROOT
mp.mp.dps = 40


# ---- 1. symphony tables --------------------------------------------------------------------------
SYMPHONY = {
    "thermal_table.csv": ["nu", "Thetae", "B", "ne", "theta", "jI", "jQ", "jV", "aI", "aQ", "aV", "rhoQ", "rhoV", "rhoV_dexter",
                          "jI_pandya", "jQ_pandya", "jV_pandya"],
    "powerlaw_table.csv": ["nu", "p", "gamma_min", "gamma_max", "B", "ne", "theta", "jI", "jQ", "jV", "aI", "aQ", "aV"],
    "kappa_table.csv": ["nu", "kappa", "w", "B", "ne", "theta", "jI", "jQ", "jV", "aI", "aQ", "aV", "rhoQ", "rhoV"],
    "powerlaw_rho_table.csv": ["nu", "B", "theta", "p", "gamma_min", "gamma_max", "ne", "rhoQ", "rhoV"],
}


def extract_symphony():
    src = os.path.join(reference_root(), "validation", "symphony")
    for name, cols in SYMPHONY.items():
        with open(os.path.join(src, name)) as f:
            rows = list(csv.DictReader(f))
        keep = rows[::4] if len(rows) > 100 else rows
        with open(os.path.join(HERE, "symphony_" + name), "w", newline="") as f:
            w = csv.writer(f)
            w.writerow(cols)
            for r in keep:
                w.writerow([r[c] for c in cols])


def extract_ipole_riaf():
    src = os.path.join(reference_root(), "validation", "ipole_riaf")
    arrays = {}
    for tag in ("fine", "2thz"):
        for st in "IQUV":
            arrays[f"{tag}_{st}"] = np.loadtxt(os.path.join(src, f"riaf_{tag}_{st}.csv"), delimiter=",", dtype=np.float64)
    np.savez_compressed(os.path.join(HERE, "ipole_riaf.npz"), **arrays)


UVFITS = ["synth_eht2017.uvfits", "synth_eht2017_noiseless.uvfits", "synth_eht2017_ehtim.csv", "synth_eht2017_noiseless_ehtim.csv",
          "synth_eht2017_image.fits"]


def copy_uvfits():
    import shutil
    dst = os.path.join(HERE, "uvfits")
    os.makedirs(dst, exist_ok=True)
    for name in UVFITS:
        shutil.copyfile(os.path.join(reference_root(), "test", "data", name), os.path.join(dst, name))


# ---- 2. geodesics in mpmath -----------------------------------------------------------------------
class HPRay:
    """BigFloat constants of one ray from the oracle's Float64 roots, Newton-polished
    (highprec_reference.jl:22-122 restated)."""

    def __init__(self, a, tho, alpha, beta):
        self.a, self.tho, self.alpha, self.beta = mp.mpf(a), mp.mpf(tho), mp.mpf(alpha), mp.mpf(beta)
        rc = oracle.ray_constants(a, tho, np.array([alpha]), np.array([beta]))[0]
        self.numreals = int(rc[2])
        self.eta = (self.alpha ** 2 - self.a ** 2) * mp.cos(self.tho) ** 2 + self.beta ** 2
        self.lam = -self.alpha * mp.sin(self.tho)
        a_, eta, lam = self.a, self.eta, self.lam
        c2 = a_ ** 2 - eta - lam ** 2
        c1 = 2 * (eta + (lam - a_) ** 2)
        c0 = -a_ ** 2 * eta
        roots = []
        for q in range(4):
            z = mp.mpc(rc[9 + 2 * q], rc[10 + 2 * q])
            for _ in range(100):
                p = ((z * z + c2) * z + c1) * z + c0
                dp = (4 * z * z + 2 * c2) * z + c1
                d = p / dp
                z -= d
                if abs(d) < mp.mpf(10) ** (-mp.mp.dps + 2) * max(abs(z), 1):
                    break
            roots.append(z)
        self.roots = roots
        if self.numreals == 4:
            r1, r2, r3, r4 = [z.real for z in roots]
            r31, r32, r41, r42 = r3 - r1, r3 - r2, r4 - r1, r4 - r2
            self.k = r32 * r41 / (r31 * r42)
            self.c = mp.sqrt(r31 * r42) / 2
            self.fo = 2 / mp.sqrt(r31 * r42) * mp.ellipf(mp.asin(mp.sqrt(r31 / r41)), self.k)
            self.rfun = lambda sn, cn: (r31 * r4 - r3 * r41 * sn * sn) / (r31 - r41 * sn * sn)
            self.r4 = r4
        elif self.numreals == 2:
            r1, r2 = roots[0].real, roots[1].real
            A = abs(roots[2] - roots[1])
            B = abs(roots[2] - roots[0])
            self.k = ((A + B) ** 2 - (r2 - r1) ** 2) / (4 * A * B)
            self.c = mp.sqrt(A * B)
            self.fo = mp.ellipf(mp.acos((A - B) / (A + B)), self.k) / mp.sqrt(A * B)
            self.rfun = lambda sn, cn: (-A * r1 + B * r2 + (A * r1 + B * r2) * cn) / (-A + B + (A + B) * cn)
        else:
            a1, a2 = abs(roots[3].imag), abs(roots[1].imag)
            b1, b2 = roots[3].real, roots[1].real
            C = mp.sqrt((a1 - a2) ** 2 + (b1 - b2) ** 2)
            D = mp.sqrt((a1 + a2) ** 2 + (b1 - b2) ** 2)
            self.k = 4 * C * D / (C + D) ** 2
            self.c = (C + D) / 2
            g0 = mp.sqrt(max((4 * a2 ** 2 - (C - D) ** 2) / ((C + D) ** 2 - 4 * a2 ** 2), 0))
            self.fo = 2 / (C + D) * mp.ellipf(mp.pi / 2 + mp.atan(g0), self.k)
            self.rfun = lambda sn, cn: -(a2 * (g0 - sn / cn) / (1 + g0 * sn / cn) + b1)
        # polar constants from the exact screen inputs
        Dth = (1 - (eta + lam ** 2) / a_ ** 2) / 2
        dsc = mp.sqrt(Dth ** 2 + eta / a_ ** 2)
        up, um = Dth + dsc, Dth - dsc
        m = up / um
        self.tempfac = 1 / mp.sqrt(abs(um * a_ ** 2))
        self.vortical = eta < 0
        sb = mp.sign(self.beta)
        ct = mp.cos(self.tho)
        if self.vortical:
            self.kth = 1 - m
            G = self.tempfac * mp.ellipf(mp.asin(mp.sqrt(min(max((ct ** 2 - um) / (up - um), 0), 1))), self.kth)
            sigma = -1 if self.tho > mp.pi / 2 else 1
            self.offset, self.sgn = sigma * sb * G, sigma
        else:
            self.kth = m
            G = self.tempfac * mp.ellipf(mp.asin(min(max(ct / mp.sqrt(up), -1), 1)), self.kth)
            self.offset, self.sgn = sb * G, sb
        self.up, self.um = up, um
        self.rp = 1 + mp.sqrt(1 - a_ ** 2)

    def coords(self, tau):
        X = self.c * (self.fo - tau)
        sn, cn = (mp.re(mp.ellipfun(f, X, m=self.k)) for f in ("sn", "cn"))
        r = mp.re(self.rfun(sn, cn))
        Xt = (tau + self.offset) / self.tempfac
        snt = mp.re(mp.ellipfun("sn", Xt, m=self.kth))
        if self.vortical:
            cth = self.sgn * mp.sqrt(self.um + (self.up - self.um) * snt ** 2)
        else:
            cth = self.sgn * mp.sqrt(self.up) * snt
        cth = min(max(cth, -1), 1)
        return r, mp.acos(cth), cth

    def rates(self, tau):
        r, th, cth = self.coords(tau)
        a, lam = self.a, self.lam
        D = r * r - 2 * r + a * a
        s2 = 1 - cth * cth
        dt = (r * r + a * a) * (r * r + a * a - a * lam) / D + a * (lam - a * s2)
        dphi = a * (2 * r - a * lam) / D + lam / s2
        return dt, dphi


GATE_SPACETIMES = [(0.94, 17.0), (0.5, 60.0), (0.7, 120.0)]


def gate_pixels(a, tho_deg, rng, n=6):
    """Random screen points of every root case plus a few near the critical curve."""
    tho = np.deg2rad(tho_deg)
    pts = []
    while len(pts) < n:
        al, be = rng.uniform(-12, 12, 2)
        pts.append((al, be))
    for psi in (0.3, 2.2, 4.0):
        # bisection for the critical screen radius along psi
        lo, hi = 1.0, 12.0
        nr = lambda rho: oracle.ray_constants(a, tho, np.array([rho * np.cos(psi)]), np.array([rho * np.sin(psi)]))[0][2]
        if nr(hi) != 4:
            continue
        for _ in range(60):
            mid = (lo + hi) / 2
            if nr(mid) == 4:
                hi = mid
            else:
                lo = mid
        for d in (1e-3, -1e-3):
            rho = hi * (1 + d)
            pts.append((rho * np.cos(psi), rho * np.sin(psi)))
    return pts


def geodesic_fixtures(N=1000, max_intervals=160):
    rng = np.random.Generator(np.random.PCG64(2024))
    out = []
    for a, tho_deg in GATE_SPACETIMES:
        tho = np.deg2rad(tho_deg)
        for al, be in gate_pixels(a, tho_deg, rng):
            ray = HPRay(a, tho, al, be)
            rc = oracle.ray_constants(a, tho, np.array([al]), np.array([be]))[0]
            tau_total, tau_valid = rc[6], rc[7]
            dtau = tau_total / (N + 1)
            ks = [1, 2, 3, N // 4, N // 3, N // 2, 2 * N // 3, 3 * N // 4, N - 1, N]
            samples = []
            for k in ks:
                tau = mp.mpf(k * dtau)
                if k * dtau > tau_valid:
                    continue
                r, th, _ = ray.coords(tau)
                samples.append({"k": k, "r": float(r), "theta": float(th)})
            # increments of t~, phi by 16-point Gauss-Legendre of the raw rates, samples inside 50 M
            xs, ws = np.polynomial.legendre.leggauss(16)
            xs = [mp.mpf(x) for x in xs]
            ws = [mp.mpf(w) for w in ws]
            inc = []
            st, sp = mp.mpf(0), mp.mpf(0)
            kfirst = None
            for k in range(1, N + 1):
                tau = mp.mpf(k * dtau)
                r, _, _ = ray.coords(tau)
                if k * dtau > tau_valid or r < ray.rp * mp.mpf(1.15):
                    break
                if kfirst is None:
                    if r <= 50:
                        kfirst = k
                        inc.append({"k": k, "dt": 0.0, "dphi": 0.0})
                    continue
                a0, b0 = mp.mpf((k - 1) * dtau), tau
                mid, half = (a0 + b0) / 2, (b0 - a0) / 2
                for x, w in zip(xs, ws):
                    dt, dp = ray.rates(mid + half * x)
                    st += half * w * dt
                    sp += half * w * dp
                if r <= 50 and k % 4 == 0:
                    inc.append({"k": k, "dt": float(st), "dphi": float(sp)})
                if k - kfirst >= max_intervals:
                    break
            out.append({"a": a, "theta_o": tho, "alpha": al, "beta": be, "N": N, "numreals": ray.numreals,
                        "samples": samples, "increments": inc})
            print(f"a={a} tho={tho_deg} ({al:.3f},{be:.3f}) case {ray.numreals}: {len(samples)} samples, {len(inc)} increments", flush=True)
    with open(os.path.join(HERE, "geodesic_pins.json"), "w") as f:
        json.dump(out, f, indent=0)


def anchor_fixtures(N=64):
    """Absolute t~ and phi at a few samples of a few rays (adaptive quadrature from the observer)."""
    out = []
    cases = [(0.94, 17.0, 5.3, 1.45), (0.94, 17.0, -2.0, 1.0), (0.5, 60.0, 7.0, -9.0), (0.5, 60.0, 1.2, 2.3)]
    for a, tho_deg, al, be in cases:
        tho = np.deg2rad(tho_deg)
        ray = HPRay(a, tho, al, be)
        rc = oracle.ray_constants(a, tho, np.array([al]), np.array([be]))[0]
        dtau = rc[6] / (N + 1)
        vals = []
        for k in (1, 5, N // 2, N - 4):
            tau = mp.mpf(k * dtau)
            tau0 = tau * mp.mpf(10) ** -14
            grid = [tau0 * mp.mpf(10) ** e for e in range(0, 15)]
            if ray.numreals == 4 and ray.fo < tau:
                grid = sorted(set([g for g in grid if g < ray.fo] + [ray.fo] + [g for g in grid if g > ray.fo]))
            grid[-1] = tau
            grid = [g for g in grid if g <= tau]
            It = mp.quad(lambda x: ray.rates(x)[0], grid)
            r0, _, _ = ray.coords(tau0)
            t_reg = It - (r0 + 2 * mp.log(r0))
            Ip = mp.quad(lambda x: ray.rates(x)[1], [mp.mpf(0)] + grid[1:])
            vals.append({"k": k, "t": float(t_reg), "phi": float(Ip)})
            print(f"anchor a={a} ({al},{be}) k={k}: t~={float(t_reg):.12f} phi={float(Ip):.12f}", flush=True)
        out.append({"a": a, "theta_o": tho, "alpha": al, "beta": be, "N": N, "values": vals})
    with open(os.path.join(HERE, "anchor_pins.json"), "w") as f:
        json.dump(out, f, indent=0)


# ---- 3. transfer step, Bessel and elliptic functions ------------------------------------------------
def step_fixtures():
    rng = np.random.Generator(np.random.PCG64(99))
    out = []
    regimes = [(1e-3, 1e-3), (0.5, 0.5), (3.0, 0.1), (0.1, 5.0), (20.0, 1.0), (1.0, 80.0), (1e-9, 1e-9), (40.0, 40.0)]
    for scale_a, scale_r in regimes:
        for _ in range(4):
            aI = abs(rng.normal()) * scale_a + 1e-12
            av = rng.normal(size=3) * scale_a * 0.4
            rv = rng.normal(size=3) * scale_r
            j = np.abs(rng.normal(size=4)) * np.array([1.0, 0.3, 0.3, 0.2])
            D = 10 ** rng.uniform(-2, 0.5)
            K = mp.matrix([[aI, av[0], av[1], av[2]], [av[0], aI, rv[2], -rv[1]], [av[1], -rv[2], aI, rv[0]], [av[2], rv[1], -rv[0], aI]])
            Aug = mp.zeros(8, 8)
            for i in range(4):
                for q in range(4):
                    Aug[i, q] = -K[i, q] * D
                Aug[i, 4 + i] = D
            E8 = mp.expm(Aug)
            O = [[float(E8[i, q]) for q in range(4)] for i in range(4)]
            Ej = [[E8[i, 4 + q] for q in range(4)] for i in range(4)]
            E = [float(sum(Ej[i][q] * j[q] for q in range(4))) for i in range(4)]
            out.append({"j": j.tolist(), "alpha": [aI] + av.tolist(), "rho": rv.tolist(), "D": D, "O": O, "E": E})
    with open(os.path.join(HERE, "step_pins.json"), "w") as f:
        json.dump(out, f, indent=0)


def special_fixtures():
    xs = [1e-3, 0.02, 0.1, 0.5, 1.0, 1.7, 3.0, 8.0, 25.0, 100.0]
    bessel = [{"x": x, "k0": float(mp.besselk(0, x)), "k1": float(mp.besselk(1, x))} for x in xs]
    ell = []
    for m in (-30.0, -3.0, -0.5, 0.0, 0.3, 0.9, 0.999, 1 - 1e-6):
        for phi in (0.1, 1.2, 2.9, 7.5):
            ell.append({"phi": phi, "m": m, "F": float(mp.ellipf(phi, m))})
    jac = []
    for m in (0.1, 0.5, 0.9, 0.99, 0.9999, 1 - 1e-7):
        for u in (0.05, 0.7, 2.3, 9.0, 21.0):
            jac.append({"u": u, "m": m, "sn": float(mp.ellipfun("sn", u, m=m)), "cn": float(mp.ellipfun("cn", u, m=m)),
                        "dn": float(mp.ellipfun("dn", u, m=m))})
    with open(os.path.join(HERE, "special_pins.json"), "w") as f:
        json.dump({"bessel": bessel, "ellipf": ell, "jacobi": jac}, f, indent=0)


if __name__ == "__main__":
    oracle.build()
    args = sys.argv[1:]
    if "--reference" in args:
        i = args.index("--reference")
        REFERENCE_ROOT = args[i + 1]
        del args[i:i + 2]
    what = args or ["symphony", "ipole", "uvfits", "special", "step", "geodesic", "anchor"]
    if "symphony" in what:
        extract_symphony()
    if "ipole" in what:
        extract_ipole_riaf()
    if "uvfits" in what:
        copy_uvfits()
    if "special" in what:
        special_fixtures()
    if "step" in what:
        step_fixtures()
    if "geodesic" in what:
        geodesic_fixtures()
    if "anchor" in what:
        anchor_fixtures()
