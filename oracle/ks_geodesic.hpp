// ks_geodesic.hpp -- CPU FP64 restatement of kerrsplat's geodesic layer (the oracle).
//
// TEST INFRASTRUCTURE ONLY. This file is the checker for the CUDA library: it is compiled into
// oracle/_build/libks_oracle.so, which only tests/, __graft_entry__.smoke() and the CPU-baseline
// leg of bench.py load. Nothing in kerrsplat_b200/ includes or links it.
//
// It follows the reference (KerrSplat.jl) line by line where the reference has code, citing
// src/Geodesics/*.jl by file:line, and restates from the published mathematics the pieces that
// the reference takes from Krang.jl @ f36f43a (absent here):
//   * radial roots: Gralla & Lupsasca 2020 (PRD 101, 044032), the resolvent-cubic solution of
//     R(r) = r^4 + (a^2 - eta - lambda^2) r^2 + 2 (eta + (lambda - a)^2) r - a^2 eta;
//   * I0_inf, G_theta^o: the closed forms of test/highprec_reference.jl:65-122 (which restates
//     Krang's _rs_case* and _theta_s);
//   * the anchors t~(tau), phi(tau) (Krang's emission_coordinates): the reference's own
//     decomposition of the Mino-time rates (quadrature.jl:1-35, three singular parts integrated in
//     closed form) with the smooth remainder integrated by 16-point Gauss-Legendre panels, the
//     regularization of t~ being the one of docs/notes/2026-09-03_phase3_slowlight.md:6-8
//     (t~ = elapsed time minus the divergent r_obs + 2 ln r_obs) and phi(0) = 0 at the observer.
//   * Jacobi amplitude: the arithmetic-geometric-mean method (DLMF 22.20(ii)); incomplete elliptic
//     integral of the first kind through Carlson's R_F (Carlson 1995, duplication theorem).
#pragma once
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <limits>
#include <vector>

namespace kso {

constexpr double PI = 3.141592653589793238462643383279502884;
constexpr double DEPS = std::numeric_limits<double>::epsilon();

// ---- elliptic building blocks -----------------------------------------------------------------

// Carlson's symmetric integral R_F(x, y, z) (Carlson 1995, Numer. Algorithms 10, 13, algorithm 1).
inline double carlson_rf(double x, double y, double z) {
    double A0 = (x + y + z) / 3.0;
    double Q = std::pow(3.0 * DEPS / 2, -1.0 / 6.0) *
               std::max({std::fabs(A0 - x), std::fabs(A0 - y), std::fabs(A0 - z)});
    double xn = x, yn = y, zn = z, An = A0, f = 1.0;
    for (int it = 0; it < 60 && f * Q >= std::fabs(An); ++it) {
        double sx = std::sqrt(xn), sy = std::sqrt(yn), sz = std::sqrt(zn);
        double lam = sx * sy + sx * sz + sy * sz;
        xn = (xn + lam) * 0.25; yn = (yn + lam) * 0.25; zn = (zn + lam) * 0.25;
        An = (An + lam) * 0.25; f *= 0.25;
    }
    double X = (A0 - x) * f / An, Y = (A0 - y) * f / An, Z = -X - Y;
    double E2 = X * Y - Z * Z, E3 = X * Y * Z;
    return (1.0 - E2 / 10.0 + E3 / 14.0 + E2 * E2 / 24.0 - 3.0 * E2 * E3 / 44.0) / std::sqrt(An);
}

// Complete integral K(m) = R_F(0, 1 - m, 1), m < 1.
inline double ellipk(double m) { return carlson_rf(0.0, 1.0 - m, 1.0); }

// Incomplete integral of the first kind F(phi | m) for any real phi (quasi-periodic unfolding
// F(phi + j pi) = F(phi) + 2 j K) and m < 1 (negative m included).
inline double ellipf(double phi, double m) {
    double j = std::nearbyint(phi / PI);
    double pr = phi - j * PI;
    double s = std::sin(pr), c = std::cos(pr);
    double F = s * carlson_rf(c * c, 1.0 - m * s * s, 1.0);
    if (j != 0.0) F += 2.0 * j * ellipk(m);
    return F;
}

// Jacobi amplitude am(u | m), 0 <= m < 1, by the AGM scale (DLMF 22.20.1-22.20.4): c_{n+1} is
// formed as c_n^2 / (4 a_{n+1}) so that it keeps relative accuracy.
inline double jacobi_am(double u, double m) {
    if (m == 0.0) return u;
    double a[12], c[12];
    a[0] = 1.0; c[0] = std::sqrt(m);
    double b = std::sqrt(1.0 - m);
    int n = 0;
    while (n < 11 && std::fabs(c[n]) > DEPS * a[n]) {
        a[n + 1] = 0.5 * (a[n] + b);
        c[n + 1] = c[n] * c[n] / (4.0 * a[n + 1]);
        b = std::sqrt(a[n] * b);
        ++n;
    }
    double phi = std::ldexp(a[n] * u, n);
    for (int i = n; i > 0; --i) phi = 0.5 * (phi + std::asin(c[i] * std::sin(phi) / a[i]));
    return phi;
}

// ---- jacobi.jl ------------------------------------------------------------------------------------

struct JState { double sn, cn, dn; };

// jacobi.jl:21-25 (amplitude, then sin/cos taken separately)
inline JState jacobi_state(double u, double mu) {
    double ph = jacobi_am(u, mu);
    double s = std::sin(ph), c = std::cos(ph);
    return {s, c, std::sqrt(std::fma(-mu, s * s, 1.0))};
}

// jacobi.jl:39-45: the addition theorems, 15 multiplications and one division
inline JState jacobi_step(const JState& x, const JState& d, double mu) {
    double den = 1.0 - mu * (x.sn * x.sn) * (d.sn * d.sn);
    double sn = (x.sn * d.cn * d.dn + d.sn * x.cn * x.dn) / den;
    double cn = (x.cn * d.cn - x.sn * x.dn * d.sn * d.dn) / den;
    double dn = (x.dn * d.dn - mu * x.sn * x.cn * d.sn * d.cn) / den;
    return {sn, cn, dn};
}

// jacobi.jl:53-56
inline JState jacobi_step_constants(double delta, double mu) {
    JState x = jacobi_state(std::fabs(delta), mu);
    return {std::copysign(x.sn, delta), x.cn, x.dn};
}

// ---- camera.jl ------------------------------------------------------------------------------------

// camera.jl:122-124: Krang's endpoint-inclusive grid axis
inline double grid_axis(double lo, double hi, int n, int i /*0-based*/) {
    if (n == 1) return lo;
    return lo + (hi - lo) * (double(i + 1) - 1.0) / double(n - 1);
}

// ---- radial roots and root cases (Gralla & Lupsasca 2020, sec. IV) -------------------------------

struct Roots { std::complex<double> r[4]; int numreals; };

inline double eta_of(double a, double alpha, double beta, double thetao) {
    double c = std::cos(thetao);
    return (alpha * alpha - a * a) * c * c + beta * beta;
}
inline double lambda_of(double alpha, double thetao) { return -alpha * std::sin(thetao); }

// Roots of R(r) with the resolvent cubic. The real/complex split is decided by the signs of the two
// inner discriminants, so r1 <= r2 and r3 <= r4 when real; numreals = 4, 2 or 0.
inline Roots radial_roots(double a, double eta, double lam) {
    using C = std::complex<double>;
    double A = a * a - eta - lam * lam;
    double B = 2.0 * (eta + (lam - a) * (lam - a));
    double Cc = -a * a * eta;
    double P = -A * A / 12.0 - Cc;
    double Q = -A / 3.0 * ((A / 6.0) * (A / 6.0) - Cc) - B * B / 8.0;
    double disc = (P / 3.0) * (P / 3.0) * (P / 3.0) + (Q / 2.0) * (Q / 2.0);
    C sq = std::sqrt(C(disc, 0.0));
    C wp = std::pow(C(-Q / 2.0, 0.0) + sq, 1.0 / 3.0);
    C wm = (std::abs(wp) > 0.0) ? C(-P / 3.0, 0.0) / wp : std::pow(C(-Q / 2.0, 0.0) - sq, 1.0 / 3.0);
    double xi0 = (wp + wm).real() - A / 3.0;
    double z = std::sqrt(std::max(xi0 / 2.0, 0.0));
    double arg12 = -A / 2.0 - z * z + B / (4.0 * z);
    double arg34 = -A / 2.0 - z * z - B / (4.0 * z);
    Roots R;
    if (arg12 >= 0.0) {
        double s = std::sqrt(arg12);
        R.r[0] = C(-z - s, 0.0); R.r[1] = C(-z + s, 0.0);
    } else {
        double s = std::sqrt(-arg12);
        R.r[0] = C(-z, -s); R.r[1] = C(-z, s);
    }
    if (arg34 >= 0.0) {
        double s = std::sqrt(arg34);
        R.r[2] = C(z - s, 0.0); R.r[3] = C(z + s, 0.0);
    } else {
        double s = std::sqrt(-arg34);
        R.r[2] = C(z, -s); R.r[3] = C(z, s);
    }
    R.numreals = (arg12 >= 0.0 ? 2 : 0) + (arg34 >= 0.0 ? 2 : 0);
    return R;
}

// Krang's radial potential R(r) and polar potential Theta(theta) (Gralla & Lupsasca eq. 7-8).
inline double r_potential(double a, double eta, double lam, double r) {
    double P = r * r + a * a - a * lam;
    double D = r * r - 2.0 * r + a * a;
    return P * P - D * (eta + (lam - a) * (lam - a));
}
inline double theta_potential(double a, double eta, double lam, double th) {
    double s = std::sin(th), c = std::cos(th);
    return eta + a * a * c * c - lam * lam * c * c / (s * s);
}

inline double horizon(double a) { return 1.0 + std::sqrt(1.0 - a * a); }

// ---- per-ray constants (pixel_constants.jl, recurrence.jl, quadrature.jl) -------------------------

enum { CASE2 = 2, CASE3 = 3, CASE4 = 4 };

struct Ray {
    // screen and spacetime
    double a, thetao, alpha, beta, eta, lam;
    Roots roots;
    int rcase;            // 2, 3, 4 (numreals 4, 2, 0)
    // radial (recurrence.jl:36-109)
    double k, c, fo;
    double r1, r3, r41, r43;          // case 2
    double n0, n1, d0, d1;            // case 3
    double a2, b1, g0;                // case 4
    double tau_valid;                 // last valid Mino time (case 2 turning inside the horizon)
    double tau_total;                 // Mino time at the horizon (plunging) or back at infinity
    // polar (recurrence.jl:196-237)
    double pmu, pscale, tempfac, poffset, sqrt_up, um, up_m_um, psign;
    bool vortical;
    double Gtheta_o;
    // quadrature constants (quadrature.jl:42-97)
    double rp, rmn, sp, sm, Qt, Qtm, Qphi, Qphim, r4q, qC, qn, sqrt_eps, gc, mp, K2;
    bool scattering;
    // visibility (recurrence.jl:285-298)
    double v_absalpha, v_alpha2, v_absbeta_eps, v_abscos, v_cos2;
};

inline double signum(double x) { return x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0); }

// Mino time at which the radial closed form reaches radius r on the inbound branch X in
// (0, X(0)): the inverse of the case's r(X) map (recurrence.jl:169-177), tau = fo - X / c.
inline double mino_time_at_radius(const Ray& R, double r) {
    double X;
    if (R.rcase == CASE2) {
        double r1 = R.roots.r[0].real(), r3 = R.roots.r[2].real(), r4 = R.roots.r[3].real();
        double r31 = r3 - r1, r41 = r4 - r1;
        double s2 = r31 * (r4 - r) / (r41 * (r3 - r));
        X = ellipf(std::asin(std::sqrt(std::max(0.0, std::min(1.0, s2)))), R.k);
    } else if (R.rcase == CASE3) {
        double cn = (R.n0 - r * R.d0) / (r * R.d1 - R.n1);
        X = ellipf(std::acos(std::max(-1.0, std::min(1.0, cn))), R.k);
    } else {
        double w = -(r + R.b1) / R.a2;
        double sc = (R.g0 - w) / (1.0 + w * R.g0);
        double ph = std::atan(sc);
        if (ph < 0.0) ph += PI;
        X = ellipf(ph, R.k);
    }
    return R.fo - X / R.c;
}

// K1 and the per-ray constants. Follows pixel_constants.jl:121-157 (with the Krang pixel restated),
// recurrence.jl:64-109 (radial marchers), 207-237 (PolarMarcher), quadrature.jl:68-97.
inline Ray make_ray(double a, double thetao, double alpha, double beta) {
    Ray R{};
    R.a = a; R.thetao = thetao; R.alpha = alpha; R.beta = beta;
    R.eta = eta_of(a, alpha, beta, thetao);
    R.lam = lambda_of(alpha, thetao);
    R.roots = radial_roots(a, R.eta, R.lam);
    int nr = R.roots.numreals;
    R.rcase = nr == 4 ? CASE2 : (nr == 2 ? CASE3 : CASE4);
    double rh = horizon(a);
    if (R.rcase == CASE2) {
        double r1 = R.roots.r[0].real(), r2 = R.roots.r[1].real(), r3 = R.roots.r[2].real(), r4 = R.roots.r[3].real();
        double r31 = r3 - r1, r32 = r3 - r2, r41 = r4 - r1, r42 = r4 - r2;
        R.k = r32 * r41 / (r31 * r42);
        R.c = std::sqrt(r31 * r42) / 2.0;
        R.fo = 2.0 / std::sqrt(r31 * r42) * ellipf(std::asin(std::sqrt(r31 / r41)), R.k);
        R.r1 = r1; R.r3 = r3; R.r41 = r41; R.r43 = r4 - r3;
        R.tau_total = 2.0 * R.fo;
        R.tau_valid = r4 < rh ? mino_time_at_radius(R, rh) : std::numeric_limits<double>::infinity();
    } else if (R.rcase == CASE3) {
        std::complex<double> z1 = R.roots.r[0], z2 = R.roots.r[1], z3 = R.roots.r[2];
        double r1 = z1.real(), r2 = z2.real();
        double r21 = (z2 - z1).real();
        double A = std::sqrt(std::norm(z3 - z2));
        double B = std::sqrt(std::norm(z3 - z1));
        R.k = ((A + B) * (A + B) - r21 * r21) / (4.0 * A * B);
        R.c = std::sqrt(A * B);
        R.fo = ellipf(std::acos((A - B) / (A + B)), R.k) / std::sqrt(A * B);
        R.n0 = -A * r1 + B * r2; R.n1 = A * r1 + B * r2; R.d0 = B - A; R.d1 = A + B;
        R.tau_valid = std::numeric_limits<double>::infinity();
        R.tau_total = mino_time_at_radius(R, rh);
    } else {
        std::complex<double> z2 = R.roots.r[1], z4 = R.roots.r[3];
        double a1 = std::fabs(z4.imag()), a2 = std::fabs(z2.imag());
        double b1 = z4.real(), b2 = z2.real();
        double C = std::sqrt((a1 - a2) * (a1 - a2) + (b1 - b2) * (b1 - b2));
        double D = std::sqrt((a1 + a2) * (a1 + a2) + (b1 - b2) * (b1 - b2));
        R.k = 4.0 * C * D / ((C + D) * (C + D));
        R.c = (C + D) / 2.0;
        R.g0 = std::sqrt(std::max((4.0 * a2 * a2 - (C - D) * (C - D)) / ((C + D) * (C + D) - 4.0 * a2 * a2), 0.0));
        R.fo = 2.0 / (C + D) * ellipf(PI / 2.0 + std::atan(R.g0), R.k);
        R.a2 = a2; R.b1 = b1;
        R.tau_valid = std::numeric_limits<double>::infinity();
        R.tau_total = mino_time_at_radius(R, rh);
    }
    // polar constants, Krang's rounding (recurrence.jl:218-236)
    double eta = R.eta, lam = R.lam;
    double Dth = (1.0 - (eta + lam * lam) / (a * a)) / 2.0;
    double dsc = std::sqrt(Dth * Dth + eta / (a * a));
    double up = Dth + dsc, um = Dth - dsc;
    double m = up / um;
    R.tempfac = 1.0 / std::sqrt(std::fabs(um * a * a));
    R.vortical = eta < 0.0;
    double sb = signum(beta);
    double ct = std::cos(thetao);
    double kq;
    if (R.vortical) {
        kq = 1.0 - m;
        double arg = std::max(0.0, std::min(1.0, (ct * ct - um) / (up - um)));
        R.Gtheta_o = R.tempfac * ellipf(std::asin(std::sqrt(arg)), kq);
        double sigma = thetao > PI / 2.0 ? -1.0 : 1.0;
        R.poffset = sigma * sb * R.Gtheta_o;
        R.psign = sigma;
    } else {
        kq = m;
        double arg = std::max(-1.0, std::min(1.0, ct / std::sqrt(up)));
        R.Gtheta_o = R.tempfac * ellipf(std::asin(arg), kq);
        R.poffset = sb * R.Gtheta_o;
        R.psign = sb;
    }
    R.pmu = -kq / (1.0 - kq);           // jacobi.jl:69-71
    R.pscale = std::sqrt(1.0 - kq);
    R.sqrt_up = std::sqrt(up); R.um = um; R.up_m_um = up - um;
    // quadrature constants (quadrature.jl:68-97)
    R.rp = 1.0 + std::sqrt(1.0 - a * a);
    R.rmn = 1.0 - std::sqrt(1.0 - a * a);
    double E = R.rp * R.rp + a * a - a * lam;
    double Em = R.rmn * R.rmn + a * a - a * lam;
    R.sp = -std::fabs(E); R.sm = -std::fabs(Em);
    R.Qt = (R.rp * R.rp + a * a) * E / (R.rp - R.rmn);
    R.Qtm = -(R.rmn * R.rmn + a * a) * Em / (R.rp - R.rmn);
    R.Qphi = a * (2.0 * R.rp - a * lam) / (R.rp - R.rmn);
    R.Qphim = -a * (2.0 * R.rmn - a * lam) / (R.rp - R.rmn);
    R.scattering = (R.rcase == CASE2) && !std::isfinite(R.tau_valid);
    R.r4q = R.rcase == CASE2 ? R.roots.r[3].real() : std::numeric_limits<double>::quiet_NaN();
    double mu_neg = -R.pmu / (1.0 - R.pmu);
    double upq = R.sqrt_up * R.sqrt_up;
    if (R.vortical) { R.qC = 1.0 / (1.0 - R.um); R.qn = (upq - R.um) / (1.0 - R.um); }
    else { R.qC = 1.0; R.qn = upq; }
    R.sqrt_eps = std::sqrt(std::max(1.0 - R.qn, 0.0));
    R.gc = 1.0 / std::sqrt(1.0 - mu_neg);
    R.mp = mu_neg / (1.0 - mu_neg);
    R.K2 = 2.0 * ellipk(R.pmu) / R.pscale;
    // visibility constants (recurrence.jl:293-298)
    R.v_absalpha = std::fabs(alpha); R.v_alpha2 = alpha * alpha;
    R.v_absbeta_eps = std::fabs(beta) + DEPS;
    R.v_abscos = std::fabs(ct); R.v_cos2 = ct * ct;
    return R;
}

// recurrence.jl:150-153
inline int anchor_interval(int M, double one_minus_k) {
    double scaled = M * std::sqrt(std::max(one_minus_k, 0.0) / 2e-5);
    double v = std::min(scaled, double(M));
    int t = int(v);   // unsafe_trunc of a non-negative finite value
    return std::max(4, std::min(M, t));
}

// direct_march.jl:45
inline double mino_step(double tau_total, int N) { return tau_total / (N + 1); }

inline double radial_argument(const Ray& R, double tau) { return R.c * (R.fo - tau); }
inline double polar_argument(const Ray& R, double tau) { return R.pscale * (tau + R.poffset) / R.tempfac; }

// recurrence.jl:169-177
inline double radius(const Ray& R, const JState& x) {
    if (R.rcase == CASE2) {
        double cn2 = R.r41 * x.cn * x.cn;
        return (R.r3 * cn2 - R.r1 * R.r43) / (cn2 - R.r43);
    } else if (R.rcase == CASE3) {
        return (R.n0 + R.n1 * x.cn) / (R.d0 + R.d1 * x.cn);
    }
    double sc = x.sn / x.cn;
    return -(R.a2 * (R.g0 - sc) / (1.0 + R.g0 * sc) + R.b1);
}

struct Polar { double theta, cos_theta; bool nu_theta; };

// recurrence.jl:248-259
inline Polar polar_angle_cos(const Ray& R, const JState& x) {
    double snX = x.sn / (R.pscale * x.dn);
    double c; bool nu;
    if (R.vortical) {
        c = R.psign * std::sqrt(std::max(R.um + R.up_m_um * snX * snX, 0.0));
        nu = R.psign * x.sn * x.cn > 0.0;
    } else {
        c = R.psign * R.sqrt_up * snX;
        nu = R.psign * x.cn > 0.0;
    }
    c = std::max(-1.0, std::min(1.0, c));
    return {std::acos(c), c, nu};
}

// recurrence.jl:299-308
inline bool krang_visible(const Ray& R, double cos_ths) {
    if (!(cos_ths > R.v_abscos)) return true;
    double c2 = cos_ths * cos_ths;
    double s2 = 1.0 - c2;
    double amin = R.a * std::sqrt(s2);
    if (!(R.v_absalpha >= amin + DEPS)) return true;
    double temp = (R.v_cos2 - c2) * (R.v_alpha2 - R.a * R.a * s2) / (c2 - 1.0);
    double bbound = std::sqrt(std::max(temp, 0.0));
    return !(R.v_absbeta_eps < bbound);
}

// ---- quadrature.jl --------------------------------------------------------------------------------

struct RayPoint { double r, theta, cos_theta; bool nur, nutheta; double s, sn, cn, gt, gphi; };

// quadrature.jl:129-142
inline void smooth_integrands(const Ray& R, double r, double cth, double s, double sn, double cn, double dn,
                              double& gt, double& gphi) {
    double a = R.a, lam = R.lam;
    double D = r * r - 2.0 * r + a * a;
    double s2 = 1.0 - cth * cth;
    double ft = (r * r + a * a) * (r * r + a * a - a * lam) / D + a * (lam - a * s2);
    double fphi = a * (2.0 * r - a * lam) / D;
    double wp = s * R.rp / (r * (r - R.rp)) / R.sp;
    double wm = s * R.rmn / (r * (r - R.rmn)) / R.sm;
    gt = ft - std::fabs(s) * (1.0 + 2.0 / r) - R.Qt * wp - R.Qtm * wm;
    double gpol = lam * R.qC * (1.0 - R.gc * dn * (1.0 - R.mp * cn * cn / 2.0)) / (1.0 - R.qn * sn * sn);
    gphi = fphi - R.Qphi * wp - R.Qphim * wm + gpol;
}

// quadrature.jl:163-173
inline RayPoint ray_point(const Ray& R, const JState& xr, const JState& xth, double tau) {
    RayPoint p;
    p.r = radius(R, xr);
    Polar pl = polar_angle_cos(R, xth);
    p.theta = pl.theta; p.cos_theta = pl.cos_theta; p.nutheta = pl.nu_theta;
    p.nur = tau < R.fo;
    p.s = (p.nur ? -1.0 : 1.0) * std::sqrt(std::max(r_potential(R.a, R.eta, R.lam, p.r), 0.0));
    p.sn = xth.sn / (R.pscale * xth.dn);
    p.cn = xth.cn / xth.dn;
    double dn = 1.0 / xth.dn;
    smooth_integrands(R, p.r, p.cos_theta, p.s, p.sn, p.cn, dn, p.gt, p.gphi);
    return p;
}

// quadrature.jl:176-180
inline RayPoint ray_point_direct(const Ray& R, double tau) {
    JState xr = jacobi_state(radial_argument(R, tau), R.k);
    JState xth = jacobi_state(polar_argument(R, tau), R.pmu);
    return ray_point(R, xr, xth, tau);
}

// quadrature.jl:184-195
inline RayPoint ray_point_turning(const Ray& R) {
    double tau = R.fo;
    JState xth = jacobi_state(polar_argument(R, tau), R.pmu);
    RayPoint p;
    p.r = R.r4q;
    Polar pl = polar_angle_cos(R, xth);
    p.theta = pl.theta; p.cos_theta = pl.cos_theta; p.nutheta = pl.nu_theta;
    p.nur = true;
    p.s = 0.0;
    p.sn = xth.sn / (R.pscale * xth.dn);
    p.cn = xth.cn / xth.dn;
    smooth_integrands(R, p.r, p.cos_theta, p.s, p.sn, p.cn, 1.0 / xth.dn, p.gt, p.gphi);
    return p;
}

// quadrature.jl:110-121
inline void polar_A(const Ray& R, double tau, double sn, double cn, double& A, double& ph) {
    double X = (tau + R.poffset) / R.tempfac;
    double nw = std::floor((X + R.K2 / 2.0) / R.K2);
    A = (std::atan(R.sqrt_eps * sn / cn) + nw * PI) / R.sqrt_eps;
    ph = std::atan(sn / cn) + nw * PI;
}
inline double polar_closed_form(const Ray& R, double tau, double sn, double cn) {
    double A, ph;
    polar_A(R, tau, sn, cn, A, ph);
    double e = R.sqrt_eps * R.sqrt_eps;
    return R.lam * R.qC * R.tempfac * R.gc * ((1.0 + R.mp * e / (2.0 * R.qn)) * A - R.mp / (2.0 * R.qn) * ph);
}

inline double simpson3(double fa, double fm, double fb, double h) { return h / 6.0 * (fa + 4.0 * fm + fb); }

// quadrature.jl:205-215
inline void interval_increment(const Ray& R, const RayPoint& pa, const RayPoint& pm, const RayPoint& pb,
                               double ta, double tb, double& It, double& Iphi) {
    double h = tb - ta;
    double ra = pa.r, rb = pb.r;
    double dFr = (rb - ra) + 2.0 * std::log(rb / ra);
    double dFp = std::log((rb - R.rp) * ra / ((ra - R.rp) * rb)) / R.sp;
    double dFm = std::log((rb - R.rmn) * ra / ((ra - R.rmn) * rb)) / R.sm;
    It = simpson3(pa.gt, pm.gt, pb.gt, h) + std::fabs(dFr) + R.Qt * dFp + R.Qtm * dFm;
    Iphi = simpson3(pa.gphi, pm.gphi, pb.gphi, h) + R.Qphi * dFp + R.Qphim * dFm +
           polar_closed_form(R, tb, pb.sn, pb.cn) - polar_closed_form(R, ta, pa.sn, pa.cn);
}

// ---- anchors: t~ and phi at arbitrary Mino times -------------------------------------------------

// 16-point Gauss-Legendre nodes and weights on [-1, 1] (Newton on P_16, computed once).
struct GL16 {
    double x[16], w[16];
    GL16() {
        const int n = 16;
        for (int i = 0; i < n; ++i) {
            double z = std::cos(PI * (i + 0.75) / (n + 0.5)), dp = 0.0;
            for (int it = 0; it < 100; ++it) {
                double p1 = 1.0, p2 = 0.0;
                for (int j = 1; j <= n; ++j) { double p3 = p2; p2 = p1; p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j; }
                dp = n * (z * p1 - p2) / (z * z - 1.0);
                double dz = p1 / dp;
                z -= dz;
                if (std::fabs(dz) < 1e-17) break;
            }
            double p1 = 1.0, p2 = 0.0;
            for (int j = 1; j <= n; ++j) { double p3 = p2; p2 = p1; p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j; }
            dp = n * (z * p1 - p2) / (z * z - 1.0);
            x[i] = z; w[i] = 2.0 / ((1.0 - z * z) * dp * dp);
        }
    }
};
inline const GL16& gl16() { static GL16 g; return g; }

// The smooth t-integrand of quadrature.jl:138 in a form without the r^2 cancellation of
// (dt/dtau) - |dr/dtau|(1 + 2/r) at large r: with P = r^2 + a^2 - a lambda, Q = eta + (lambda - a)^2,
// sqrt(R) = |s|, the difference is Delta Q/(P + |s|) (1 + 2/r) + 2(2r - a^2) P/(r Delta).
inline double gt_large_r(const Ray& R, double r, double cth, double s) {
    double a = R.a, lam = R.lam;
    double D = r * r - 2.0 * r + a * a;
    double P = r * r + a * a - a * lam;
    double Qv = R.eta + (lam - a) * (lam - a);
    double as = std::fabs(s);
    double diff = D * Qv / (P + as) * (1.0 + 2.0 / r) + 2.0 * (2.0 * r - a * a) * P / (r * D);
    double s2 = 1.0 - cth * cth;
    double wp = s * R.rp / (r * (r - R.rp)) / R.sp;
    double wm = s * R.rmn / (r * (r - R.rmn)) / R.sm;
    return diff + a * (lam - a * s2) - R.Qt * wp - R.Qtm * wm;
}

constexpr double LARGE_R = 64.0;

// Smooth integrands at tau from the direct (non-recurrence) Jacobi states.
inline void smooth_at(const Ray& R, double tau, double& gt, double& gphi, double& r) {
    RayPoint p = ray_point_direct(R, tau);
    r = p.r;
    gt = p.gt; gphi = p.gphi;
    double P = r * r + R.a * R.a - R.a * R.lam;
    if (r > LARGE_R && P > 0.0) gt = gt_large_r(R, r, p.cos_theta, p.s);
}

// Closed-form parts of t~ and phi at tau: the large-r piece (regularized), the two horizon pieces
// and the polar piece (quadrature.jl:11-31, 208-213) accumulated from the observer (tau = 0).
inline void closed_parts(const Ray& R, double tau, double& tc, double& phic) {
    RayPoint p = ray_point_direct(R, tau);
    double r = p.r;
    double F = r + 2.0 * std::log(r);
    double L;
    if (R.scattering && tau > R.fo) {
        double F4 = R.r4q + 2.0 * std::log(R.r4q);
        L = F - 2.0 * F4;
    } else {
        L = -F;
    }
    double lp = std::log((r - R.rp) / r) / R.sp;
    double lm = std::log((r - R.rmn) / r) / R.sm;
    tc = L + R.Qt * lp + R.Qtm * lm;
    // polar closed form relative to the observer
    JState x0 = jacobi_state(polar_argument(R, 0.0), R.pmu);
    double sn0 = x0.sn / (R.pscale * x0.dn), cn0 = x0.cn / x0.dn;
    phic = R.Qphi * lp + R.Qphim * lm + polar_closed_form(R, tau, p.sn, p.cn) - polar_closed_form(R, 0.0, sn0, cn0);
}

// Integral of the smooth integrands over [ta, tb] by one 16-point Gauss-Legendre panel.
inline void gl_panel(const Ray& R, double ta, double tb, double& It, double& Iphi) {
    const GL16& g = gl16();
    double mid = 0.5 * (ta + tb), half = 0.5 * (tb - ta);
    double st = 0.0, sp = 0.0;
    for (int i = 0; i < 16; ++i) {
        double gt, gp, r;
        smooth_at(R, mid + half * g.x[i], gt, gp, r);
        st += g.w[i] * gt; sp += g.w[i] * gp;
    }
    It = half * st; Iphi = half * sp;
}

// Integral of the smooth integrands over [ta, tb] split into `npanel` panels and at the radial
// turning point of a scattering ray (where |dr/dtau| has a kink).
inline void smooth_integral(const Ray& R, double ta, double tb, int npanel, double& It, double& Iphi) {
    It = 0.0; Iphi = 0.0;
    double h = (tb - ta) / npanel;
    for (int q = 0; q < npanel; ++q) {
        double a0 = ta + q * h, b0 = (q == npanel - 1) ? tb : ta + (q + 1) * h;
        double t1, p1;
        if (R.scattering && a0 < R.fo && R.fo < b0) {
            gl_panel(R, a0, R.fo, t1, p1); It += t1; Iphi += p1;
            gl_panel(R, R.fo, b0, t1, p1); It += t1; Iphi += p1;
        } else {
            gl_panel(R, a0, b0, t1, p1); It += t1; Iphi += p1;
        }
    }
}

struct Anchor { double t, phi; bool ok; JState xr, xth; };

// Samples per Gauss-Legendre panel between anchors.
constexpr int ANCHOR_PANEL_SAMPLES = 4;

// The anchors of one ray: at samples k = 1 + m * Manchor (1-based), the states of the recurrence,
// t~, phi and Krang's validity flag (direct_march.jl:59-62 / quadrature.jl:245-291).
inline std::vector<Anchor> ray_anchors(const Ray& R, int N, int Manchor, double dtau) {
    std::vector<Anchor> out;
    double tacc = 0.0, pacc = 0.0;   // integral of the smooth parts from tau = 0
    double tprev = 0.0;
    for (int k = 1; k <= N; k += Manchor) {
        double tau = k * dtau;
        Anchor A{};
        A.xr = jacobi_state(radial_argument(R, tau), R.k);
        A.xth = jacobi_state(polar_argument(R, tau), R.pmu);
        Polar pl = polar_angle_cos(R, A.xth);
        A.ok = (tau <= R.tau_valid) && krang_visible(R, pl.cos_theta);
        bool integrable = tau <= R.tau_valid;
        if (integrable) {
            int nsamp = (k == 1) ? 1 : Manchor;
            int np = (k == 1) ? 1 : (nsamp + ANCHOR_PANEL_SAMPLES - 1) / ANCHOR_PANEL_SAMPLES;
            double It, Ip;
            smooth_integral(R, tprev, tau, np, It, Ip);
            tacc += It; pacc += Ip;
            double tc, pc;
            closed_parts(R, tau, tc, pc);
            A.t = tacc + tc;
            A.phi = pacc + pc;
        } else {
            A.t = 0.0; A.phi = 0.0;
        }
        tprev = tau;
        out.push_back(A);
    }
    return out;
}

// ---- the sample stream of march_ray (quadrature.jl:231-296) -------------------------------------

struct Sample { double t, r, theta, phi; bool nur, nutheta, ok; };

// March one ray and call f(k, sample) for k = 1..N; returns the largest anchor residuals.
template <class F>
inline void march_ray(const Ray& R, int N, int M, F&& f, double* resid_t = nullptr, double* resid_phi = nullptr) {
    double dtau = mino_step(R.tau_total, N);
    double h = dtau / 2.0;
    double tau_valid = R.tau_valid;
    int Manchor = anchor_interval(M, 1.0 - R.k);
    std::vector<Anchor> anchors = ray_anchors(R, N, Manchor, dtau);
    JState dr = jacobi_step_constants(-R.c * h, R.k);
    JState dth = jacobi_step_constants(R.pscale * h / R.tempfac, R.pmu);
    JState xr = anchors[0].xr, xth = anchors[0].xth;
    RayPoint pa = ray_point(R, xr, xth, dtau);
    double t = anchors[0].t, phi = anchors[0].phi;
    double rt = 0.0, rphi = 0.0;
    f(1, Sample{t, pa.r, pa.theta, phi, pa.nur, pa.nutheta, (dtau <= tau_valid) && krang_visible(R, pa.cos_theta)});
    for (int k = 2; k <= N; ++k) {
        double ta = (k - 1) * dtau, tb = k * dtau;
        xr = jacobi_step(xr, dr, R.k);
        xth = jacobi_step(xth, dth, R.pmu);
        RayPoint pm = ray_point(R, xr, xth, ta + h);
        bool anchor = (k - 1) % Manchor == 0;
        const Anchor* A = anchor ? &anchors[(k - 1) / Manchor] : nullptr;
        if (anchor) { xr = A->xr; xth = A->xth; }
        else { xr = jacobi_step(xr, dr, R.k); xth = jacobi_step(xth, dth, R.pmu); }
        RayPoint pb = ray_point(R, xr, xth, tb);
        if (R.scattering && ta < R.fo && R.fo < tb) {
            RayPoint pt = ray_point_turning(R);
            RayPoint p1 = ray_point_direct(R, (ta + R.fo) / 2.0);
            RayPoint p2 = ray_point_direct(R, (R.fo + tb) / 2.0);
            double It1, Ip1, It2, Ip2;
            interval_increment(R, pa, p1, pt, ta, R.fo, It1, Ip1);
            interval_increment(R, pt, p2, pb, R.fo, tb, It2, Ip2);
            t += It1 + It2; phi += Ip1 + Ip2;
        } else {
            double It, Ip;
            interval_increment(R, pa, pm, pb, ta, tb, It, Ip);
            t += It; phi += Ip;
        }
        if (anchor && A->ok) {
            rt = std::max(rt, std::fabs(t - A->t));
            rphi = std::max(rphi, std::fabs(phi - A->phi));
            t = A->t; phi = A->phi;
        }
        f(k, Sample{t, pb.r, pb.theta, phi, pb.nur, pb.nutheta, (tb <= tau_valid) && krang_visible(R, pb.cos_theta)});
        pa = pb;
    }
    if (resid_t) *resid_t = rt;
    if (resid_phi) *resid_phi = rphi;
}

// ---- coordinates.jl:22-31 ---------------------------------------------------------------------

inline void quasi_cartesian_kerr_schild(double a, double r, double th, double ph, double& x, double& y, double& z) {
    double temp = std::sqrt(1.0 - a * a);
    double rp = 1.0 + temp, rm = 1.0 - temp;
    double phks = ph + a / (2.0 * temp) * std::log(std::fabs((r - rp + DEPS) / (r - rm + DEPS))) - std::atan2(a, r);
    double st = std::sin(th), ct = std::cos(th);
    double sp = std::sin(phks), cp = std::cos(phks);
    x = r * st * cp; y = r * st * sp; z = r * ct;
}

}  // namespace kso
