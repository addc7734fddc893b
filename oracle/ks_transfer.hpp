// ks_transfer.hpp -- CPU FP64 restatement of kerrsplat's transfer layer and splat consumers (the
// oracle). TEST INFRASTRUCTURE ONLY: see ks_geodesic.hpp for who may load it.
//
// Follows, by file:line, src/Transfer/{constants,bessel,coefficients,kappa,frames,step,transport}.jl
// and src/Splats/{Splats,polarized,populations,trajectories}.jl. The Kerr metric helpers the
// reference takes from Krang (metric_uu, the ZAMO tetrad and its inverse, p_bl_d) are the textbook
// Boyer-Lindquist expressions, with Krang's ZAMO spatial axes ordered (r, phi, -theta) as
// frames.jl:7-9 states. K0 and K1 are evaluated from the integral representation
// K_nu(x) = int_0^inf exp(-x cosh t) cosh(nu t) dt by the trapezoidal rule (exponentially
// convergent for this analytic, doubly-exponentially decaying integrand); the reference uses the
// minimax fits of Bessels.jl, and both are accurate to a few ulp.
#pragma once
#include "ks_geodesic.hpp"
#include <array>

namespace kso {

// constants.jl:3-12 (ipole / symphony cgs values)
constexpr double ME = 9.1093826e-28, MP = 1.67262171e-24, CL = 2.99792458e10, EE = 4.80320680e-10;
constexpr double HPL = 6.6260693e-27, KBOL = 1.3806505e-16, GNEWT = 6.6742e-8, MSUN = 1.989e33;
constexpr double PC = 3.085678e18, JY = 1e-23;
// coefficients.jl:299-303
constexpr double NU0 = 1e11;
inline double planck0() { return 2.0 * HPL * NU0 * NU0 * NU0 / (CL * CL); }
inline double nuhat(double nu) { return nu / NU0; }

inline double gravitational_radius(double Msun) { return GNEWT * Msun * MSUN / (CL * CL); }

// ---- Bessel K0, K1 ------------------------------------------------------------------------------
inline void besselk01(double x, double& k0, double& k1) {
    // trapezoid in t on exp(-x (cosh t - 1)) (the factor exp(-x) applied at the end); the step
    // resolves the Gaussian core of width 1/std::sqrt(x) (error ~ exp(-2 pi^2 / (x h^2)) < 1e-17)
    const double h = std::fmin(0.125, 0.6 / std::sqrt(x));
    double s0 = 0.5, s1 = 0.5;
    for (int j = 1; j < 20000; ++j) {
        double t = j * h;
        double ch = std::cosh(t);
        double e = std::exp(-x * (ch - 1.0));
        s0 += e;
        s1 += e * ch;
        if (e < 1e-18 * s0) break;
    }
    double ex = std::exp(-x);
    k0 = h * s0 * ex; k1 = h * s1 * ex;
}
// coefficients.jl:79-84
inline void besselk012(double x, double& k0, double& k1, double& k2) {
    besselk01(x, k0, k1);
    k2 = k0 + 2.0 * k1 / x;
}

// coefficients.jl:50-61
inline double planck(double nu, double Te) {
    double x = HPL * nu / (ME * CL * CL * Te);
    double nh = nuhat(nu);
    double pref = planck0() * nh * nh * nh;
    if (x < 2e-3) return pref / (x / 24.0 * (24.0 + x * (12.0 + x * (4.0 + x))));
    return pref / (std::exp(x) - 1.0);
}

struct Coeffs { double jI, jQ, jV, aI, aQ, aV, rQ, rV; };

// coefficients.jl:87-89 (Dexter 2016 appendix A fits)
inline double dexter_II(double x) { return 2.5651 * (1 + 1.92 * std::pow(x, -1.0 / 3) + 0.9977 * std::pow(x, -2.0 / 3)) * std::exp(-1.8899 * std::pow(x, 1.0 / 3)); }
inline double dexter_IQ(double x) { return 2.5651 * (1 + 0.93193 * std::pow(x, -1.0 / 3) + 0.499873 * std::pow(x, -2.0 / 3)) * std::exp(-1.8899 * std::pow(x, 1.0 / 3)); }
inline double dexter_IV(double x) { return (1.81384 / x + 3.42319 * std::pow(x, -2.0 / 3) + 0.0292545 * std::pow(x, -0.5) + 2.03773 * std::pow(x, -1.0 / 3)) * std::exp(-1.8899 * std::pow(x, 1.0 / 3)); }

// coefficients.jl:147-169: Pandya et al. (2016) thermal emissivities (symphony maxwell_juettner_I/Q/V,
// ipole's signs), ipole's `emission_type 1`.
inline void thermal_synchrotron_pandya(double ne, double Te, double B, double nu, double th, double& jI, double& jQ, double& jV) {
    double st = std::sin(th);
    double nuc = EE * B / (2 * PI * ME * CL);
    double nus = (2.0 / 9.0) * nuc * st * Te * Te;
    double X = nu / nus;
    double pref = ne * EE * EE * nuc / CL;
    double term1 = std::sqrt(2.0) * PI / 27 * st;
    double x13 = std::pow(X, 1.0 / 3), x16 = std::pow(X, 1.0 / 6), x12 = std::pow(X, 0.5);
    double c1112 = std::pow(2.0, 11.0 / 12);
    double ex = std::exp(-x13);
    double bi = x12 + c1112 * x16;
    jI = pref * term1 * bi * bi * ex;
    double te = std::pow(Te, 24.0 / 25);
    double t2 = (7 * te + 35) / (10 * te + 75);
    double bq = x12 + t2 * c1112 * x16;
    jQ = pref * term1 * bq * bq * ex;
    double tv1 = (37 - 87 * std::sin(th - 28.0 / 25)) / (100 * (Te + 1));
    double tv2 = std::pow(1 + (std::pow(Te, 3.0 / 5) / 25 + 7.0 / 10) * std::pow(X, 9.0 / 25), 5.0 / 3);
    jV = pref * tv1 * tv2 * ex;
}

// coefficients.jl:101-145 (default prescription: Dexter emissivities, Shcherbakov rho_V; `pandya`
// switches the emissivities to the Pandya fits, coefficients.jl:134-135)
inline Coeffs thermal_synchrotron(double ne, double Te, double B, double nu, double th, bool dexter_rhoV = false, bool pandya = false) {
    double st = std::sin(th), ct = std::cos(th);
    double w0 = EE * B / (ME * CL);
    double wp2 = 4 * PI * ne * EE * EE / ME;
    double w = 2 * PI * nu;
    double w0w = w0 / w, wp2w2 = wp2 / (w * w);
    double k0, k1, k2;
    besselk012(1.0 / Te, k0, k1, k2);
    if (!(st > 0)) {
        double f0 = k2 > 0 ? k0 / k2 : 1.0;
        double rV0 = w / CL * (wp2w2 * w0w * f0 * ct);
        return {0, 0, 0, 0, 0, 0, 0, rV0};
    }
    double x = Te * std::sqrt(std::sqrt(2.0) * st * (1e3 * w0w));
    double extraterm = (0.011 * std::exp(-x / 47.2) - std::pow(2.0, -1.0 / 3) / std::pow(3.0, 23.0 / 6) * PI * 1e4 * std::pow(x + 1e-16, -8.0 / 3)) *
                       (0.5 + 0.5 * std::tanh((std::log(x) - std::log(120.0)) / 0.1));
    double jffunc = 2.011 * std::exp(-std::pow(x, 1.035) / 4.7) - std::cos(x / 2) * std::exp(-std::pow(x, 1.2) / 2.73) - 0.011 * std::exp(-x / 47.2) + extraterm;
    double kratio = k2 > 0 ? k1 / k2 : 1.0;
    double eps11m22 = jffunc * wp2w2 * w0w * w0w * (kratio + 6 * Te) * st * st;
    double rQ = w / (2 * CL) * eps11m22;
    double ff;
    if (dexter_rhoV && k2 > 0) ff = (k0 - 0.43793091 * std::log(1 + 0.00185777 * std::pow(x, 1.50316886))) / k2;
    else ff = (k2 > 0 ? k0 / k2 : 1.0) * (1 - 0.11 * std::log(1 + 0.035 * x));
    double rV = w / CL * (wp2w2 * w0w * ff * ct);
    double jI, jQ, jV;
    if (pandya) {
        thermal_synchrotron_pandya(ne, Te, B, nu, th, jI, jQ, jV);
    } else {
        double nus = 3 * EE * B * st / (4 * PI * ME * CL) * Te * Te + 1;
        double xs = nu / nus;
        double pref = ne * EE * EE * nu / (2 * std::sqrt(3.0) * CL * Te * Te);
        jI = pref * dexter_II(xs);
        jQ = pref * dexter_IQ(xs);
        jV = 2 * ne * EE * EE * nu * ct / st / (3 * std::sqrt(3.0) * CL * Te * Te * Te) * dexter_IV(xs);
    }
    double Bn = planck(nu, Te);
    double invB = Bn > 0 ? 1.0 / Bn : 0.0;
    return {jI, jQ, jV, jI * invB, jQ * invB, jV * invB, rQ, rV};
}

// coefficients.jl:208-218 (Jones & O'Dell rotativities)
inline void powerlaw_rotativities(double ne, double p, double gmin, double gmax, double B, double nu, double th, double& rQ, double& rV) {
    double st = std::sin(th), ct = std::cos(th);
    double nB = EE * B * st / (2 * PI * ME * CL);
    double rperp = ne * EE * EE * (p - 1) / (ME * CL * nB * (std::pow(gmin, 1 - p) - std::pow(gmax, 1 - p)));
    double nmin = gmin * gmin * nB;
    rQ = -rperp * std::pow(nB / nu, 3) * std::pow(gmin, 2 - p) * (1 - std::pow(nmin / nu, p / 2 - 1)) / (p / 2 - 1);
    rV = 2 * (p + 2) / (p + 1) * rperp * std::pow(nB / nu, 2) * std::pow(gmin, -(p + 1)) * std::log(gmin) * ct / st;
}

// coefficients.jl:235-256 (Pandya+ 2016 power-law fits)
inline Coeffs powerlaw_synchrotron(double ne, double p, double gmin, double gmax, double B, double nu, double th) {
    double st = std::sin(th), ct = std::cos(th);
    double nc = EE * B / (2 * PI * ME * CL);
    double gspan = std::pow(gmin, 1 - p) - std::pow(gmax, 1 - p);
    double pref = ne * EE * EE * nc / CL;
    double jI = pref * (std::pow(3.0, p / 2) * (p - 1) * st) / (2 * (p + 1) * gspan) *
                std::tgamma((3 * p - 1) / 12) * std::tgamma((3 * p + 19) / 12) * std::pow(nu / (nc * st), -(p - 1) / 2);
    double jQ = (p + 1) / (p + 7.0 / 3) * jI;
    double jV = (171.0 / 250) * std::pow(p, 49.0 / 100) * ct / st * std::pow(nu / (3 * nc * st), -0.5) * jI;
    double apref = ne * EE * EE / (nu * ME * CL);
    double aI = apref * std::pow(3.0, (p + 1) / 2) * (p - 1) / (4 * gspan) *
                std::tgamma((3 * p + 2) / 12) * std::tgamma((3 * p + 22) / 12) * std::pow(nu / (nc * st), -(p + 2) / 2);
    double aQ = aI * std::pow((17.0 / 500) * p - 43.0 / 1250, 43.0 / 500);
    double term6 = std::pow((31.0 / 10) * std::pow(st, -48.0 / 25) - 31.0 / 10, 64.0 / 125);
    double aV = aI * std::pow((71.0 / 100) * p + 22.0 / 625, 197.0 / 500) * term6 * std::pow(nu / (nc * st), -0.5) * signum(ct);
    double rQ, rV;
    powerlaw_rotativities(ne, p, gmin, gmax, B, nu, th, rQ, rV);
    return {jI, jQ, jV, aI, aQ, aV, rQ, rV};
}

// kappa.jl:158-180 (Marszewski+ 2021 fits at kappa = 3.5, 4, 4.5, 5)
inline double kappa_rhoQ_fit(int i, double w, double X) {
    double sw = std::sqrt(w), e5 = std::exp(-5 * w);
    if (i == 1) return (17 * w - 3 * sw + 7 * sw * e5) * (1 - std::exp(-std::pow(X, 0.84) / 30) - std::sin(X / 10) * std::exp(-3 * std::pow(X, 0.471) / 2));
    if (i == 2) return (46 * w / 3 - 5 * sw / 3 + 17 * sw / 3 * e5) * (1 - std::exp(-std::pow(X, 0.84) / 18) - std::sin(X / 6) * std::exp(-7 * std::pow(X, 0.5) / 4));
    if (i == 3) return (14 * w - 13 * sw / 8 + 9 * sw / 2 * e5) * (1 - std::exp(-std::pow(X, 0.84) / 12) - std::sin(X / 4) * std::exp(-2 * std::pow(X, 0.525)));
    return (25 * w / 2 - sw + 5 * sw * e5) * (1 - std::exp(-std::pow(X, 0.84) / 8) - std::sin(3 * X / 8) * std::exp(-9 * std::pow(X, 0.541) / 4));
}
inline double kappa_rhoV_fit(int i, double w, double X) {
    if (i == 1) return (w * w + 2 * w + 1) / (25 * w * w / 8 + 4 * w + 1) * (1 - 0.17 * std::log(1 + 0.447 * std::pow(X, -0.5)));
    if (i == 2) return (w * w + 54 * w + 50) / (30 * w * w / 11 + 134 * w + 50) * (1 - 0.17 * std::log(1 + 0.391 * std::pow(X, -0.5)));
    if (i == 3) return (w * w + 43 * w + 38) / (7 * w * w / 3 + 185 * w / 2 + 38) * (1 - 0.17 * std::log(1 + 0.348 * std::pow(X, -0.5)));
    return (w + 13.0 / 14) / (2 * w + 13.0 / 14) * (1 - 0.17 * std::log(1 + 0.313 * std::pow(X, -0.5)));
}
// kappa.jl:188-203
inline void kappa_rotativities(double ne, double kap, double w, double B, double nu, double th, double& rQ, double& rV) {
    double st = std::sin(th), ct = std::cos(th);
    double nc = EE * B / (2 * PI * ME * CL);
    double X = nu / ((w * kap) * (w * kap) * nc * st);
    double kc = std::max(3.5, std::min(5.0, kap));
    int i = kc < 4 ? 1 : (kc < 4.5 ? 2 : 3);
    double klo = 3.5 + (i - 1) / 2.0, f = (kc - klo) * 2;
    double fQ = (1 - f) * kappa_rhoQ_fit(i, w, X) + f * kappa_rhoQ_fit(i + 1, w, X);
    double fV = (1 - f) * kappa_rhoV_fit(i, w, X) + f * kappa_rhoV_fit(i + 1, w, X);
    double k0, k1, k2;
    besselk012(1.0 / w, k0, k1, k2);
    rQ = -(ne * EE * EE * nc * nc * st * st) / (ME * CL * nu * nu * nu) * fQ;
    rV = 2 * (ne * EE * EE * nc * ct) / (ME * CL * nu * nu) * (k0 / (k2 + 1e-40)) * fV;
}
// kappa.jl:109-155 (Pandya+ 2016 kappa fits, guard on |N_high| as the reference writes it)
inline Coeffs kappa_synchrotron(double ne, double kap, double w, double B, double nu, double th, double hyp) {
    double st = std::sin(th), ct = std::cos(th);
    double nc = EE * B / (2 * PI * ME * CL);
    double nw = (w * kap) * (w * kap) * nc * st;
    double X = nu / nw;
    const double small = 1e-40;
    double pref = ne * EE * EE * nc * st / CL;
    double g43 = std::tgamma(kap - 4.0 / 3), g2 = std::tgamma(kap - 2);
    double gq = std::tgamma(kap / 4 - 1.0 / 3), gp = std::tgamma(kap / 4 + 4.0 / 3);
    double NlowI = 4 * PI * g43 / (std::pow(3.0, 7.0 / 3) * g2);
    double NhighI = 0.25 * std::pow(3.0, (kap - 1) / 2) * (kap - 2) * (kap - 1) * gq * gp + small;
    double xI = 3 * std::pow(kap, -1.5);
    double jI = pref * NlowI * std::pow(X, 1.0 / 3) * std::pow(1 + std::pow(X, xI * (3 * kap - 4) / 6) * std::pow(NlowI / NhighI, xI), -1 / xI);
    double NlowQ = -0.5 * 4 * PI * g43 / (std::pow(3.0, 7.0 / 3) * g2);
    double NhighQ = -(0.8 * 0.8 + kap / 50) * 0.25 * std::pow(3.0, (kap - 1) / 2) * (kap - 2) * (kap - 1) * gq * gp + small;
    double xQ = 3.7 * std::pow(kap, -1.6);
    double jQ = -(pref * NlowQ * std::pow(X, 1.0 / 3) * std::pow(1 + std::pow(X, xQ * (3 * kap - 4) / 6) * std::pow(NlowQ / NhighQ, xQ), -1 / xQ));
    double NlowV = -(0.75 * 0.75) * std::pow(std::pow(st, -12.0 / 5) - 1, 12.0 / 25) * (std::pow(kap, -66.0 / 125) / w) * std::pow(X, -7.0 / 20) * 4 * PI * g43 / (std::pow(3.0, 7.0 / 3) * g2);
    double NhighV = -(7.0 / 8) * (7.0 / 8) * std::pow(std::pow(st, -2.5) - 1, 11.0 / 25) * (std::pow(kap, -11.0 / 25) / w) * std::pow(X, -0.5) * 0.25 * std::pow(3.0, (kap - 1) / 2) * (kap - 2) * (kap - 1) * gq * gp - small;
    double xV = 3 * std::pow(kap, -1.5);
    double jV = std::fabs(NhighV) < small * small ? 0.0
              : -(pref * NlowV * std::pow(X, 1.0 / 3) * std::pow(1 + std::pow(X, xV * (3 * kap - 4) / 6) * std::pow(NlowV / NhighV, xV), -1 / xV)) * signum(ct);
    double apref = ne * EE / (B * st);
    double g53 = std::tgamma(5.0 / 3), gk2 = std::tgamma(2 + kap / 2);
    double ck = (kap - 2) * (kap - 1) * kap;
    double NlowA = std::pow(3.0, 1.0 / 6) * (10.0 / 41) * (2 * PI) * (2 * PI) / std::pow(w * kap, 16.0 / 3 - kap) * ck / (3 * kap - 1) * g53 * hyp;
    double NhighA = 2 * std::pow(PI, 2.5) / 3 * ck / std::pow(w * kap, 5) * (2 * gk2 / (2 + kap) - 1) * (std::pow(3 / kap, 19.0 / 4) + 3.0 / 5) + small;
    double xA = std::pow(-7.0 / 4 + 8 * kap / 5, -43.0 / 50);
    double aI = apref * NlowA * std::pow(X, -5.0 / 3) * std::pow(1 + std::pow(X, xA * (3 * kap - 1) / 6) * std::pow(NlowA / NhighA, xA), -1 / xA);
    double NlowQA = -(25.0 / 48) * std::pow(3.0, 1.0 / 6) * (10.0 / 41) * (2 * PI) * (2 * PI) / std::pow(w * kap, 16.0 / 3 - kap) * ck / (3 * kap - 1) * g53 * hyp;
    double NhighQA = -(21.0 * 21.0 * std::pow(kap, -144.0 / 25) + 11.0 / 20) * 2 * std::pow(PI, 2.5) / 3 * ck / std::pow(w * kap, 5) * (2 * gk2 / (2 + kap) - 1) + small;
    double xQA = 1.4 * std::pow(kap, -23.0 / 20);
    double aQ = -(apref * NlowQA * std::pow(X, -5.0 / 3) * std::pow(1 + std::pow(X, xQA * (3 * kap - 1) / 6) * std::pow(NlowQA / NhighQA, xQA), -1 / xQA));
    double NlowVA = -(77 / (100 * w)) * std::pow(std::pow(st, -114.0 / 50) - 1, 223.0 / 500) * std::pow(X, -7.0 / 20) * std::pow(kap, -0.7) * std::pow(3.0, 1.0 / 6) * (10.0 / 41) * (2 * PI) * (2 * PI) /
                    std::pow(w * kap, 16.0 / 3 - kap) * ck / (3 * kap - 1) * g53 * hyp;
    double NhighVA = -(14.3 * std::pow(w, -116.0 / 125)) * std::pow(std::pow(st, -41.0 / 20) - 1, 0.5) * (169.0 * std::pow(kap, -8) + 13.0 / 2500 * kap - 263.0 / 5000 + 47 / (200 * kap)) *
                     std::pow(X, -0.5) * 2 * std::pow(PI, 2.5) / 3 * ck / std::pow(w * kap, 5) * (2 * gk2 / (2 + kap) - 1) + small;
    double xVA = 1.22 * std::pow(kap, -142.0 / 125) + 7.0 / 1000;
    double aV = -(apref * NlowVA * std::pow(X, -5.0 / 3) * std::pow(1 + std::pow(X, xVA * (3 * kap - 1) / 6) * std::pow(NlowVA / NhighVA, xVA), -1 / xVA)) * signum(ct);
    double rQ, rV;
    kappa_rotativities(ne, kap, w, B, nu, th, rQ, rV);
    return {jI, jQ, jV, aI, aQ, aV, rQ, rV};
}

// step.jl:57-62
inline double pow2_below(double v) {
    if (!(std::isfinite(v) && v > 0)) return 1.0;
    int e; std::frexp(v, &e);
    return std::ldexp(1.0, e - 1);
}

// coefficients.jl:264-288
inline double cap_factor(double I, double Q, double V, double fmax) {
    if (!(I > 0)) return (Q == 0.0 && V == 0.0) ? 1.0 : 0.0;
    double s = pow2_below(std::max({std::fabs(I), std::fabs(Q), std::fabs(V)}));
    double Ih = I / s, q = Q / s, v = V / s;
    double qv = q * q + v * v;
    double p = qv > 0 ? std::sqrt(qv) : 0.0;
    return p > fmax * Ih ? fmax * Ih / p : 1.0;
}
inline Coeffs cap_polarization(const Coeffs& c, double fmax = 0.99) {
    double fe = cap_factor(c.jI, c.jQ, c.jV, fmax);
    double fa = cap_factor(c.aI, c.aQ, c.aV, fmax);
    return {c.jI, fe * c.jQ, fe * c.jV, c.aI, fa * c.aQ, fa * c.aV, c.rQ, c.rV};
}
// coefficients.jl:310-314
inline Coeffs invariants(const Coeffs& c, double nu) {
    double nh = nuhat(nu);
    double i2 = 1.0 / (nh * nh);
    return {c.jI * i2, c.jQ * i2, c.jV * i2, nh * c.aI, nh * c.aQ, nh * c.aV, nh * c.rQ, nh * c.rV};
}

// ---- frames.jl --------------------------------------------------------------------------------

using M4 = std::array<double, 16>;   // row-major 4x4
using V4 = std::array<double, 4>;

inline V4 mv(const M4& A, const V4& x) {
    V4 y{};
    for (int i = 0; i < 4; ++i) y[i] = A[4 * i] * x[0] + A[4 * i + 1] * x[1] + A[4 * i + 2] * x[2] + A[4 * i + 3] * x[3];
    return y;
}
inline M4 mm(const M4& A, const M4& B) {
    M4 C{};
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            double s = 0;
            for (int k = 0; k < 4; ++k) s += A[4 * i + k] * B[4 * k + j];
            C[4 * i + j] = s;
        }
    return C;
}

// Krang's metric_uu: the inverse Boyer-Lindquist metric, (t, r, theta, phi).
inline M4 metric_uu(double a, double r, double th) {
    double s = std::sin(th), c = std::cos(th);
    double S = r * r + a * a * c * c, D = r * r - 2 * r + a * a;
    double A = (r * r + a * a) * (r * r + a * a) - a * a * D * s * s;
    M4 g{};
    g[0] = -A / (S * D);
    g[3] = g[12] = -2 * a * r / (S * D);
    g[5] = D / S;
    g[10] = 1.0 / S;
    g[15] = (D - a * a * s * s) / (S * D * s * s);
    return g;
}
// Krang's metric_dd: the Boyer-Lindquist metric, (t, r, theta, phi).
inline M4 metric_dd(double a, double r, double th) {
    double s = std::sin(th), c = std::cos(th);
    double S = r * r + a * a * c * c, D = r * r - 2 * r + a * a;
    M4 g{};
    g[0] = -(1 - 2 * r / S);
    g[3] = g[12] = -2 * a * r * s * s / S;
    g[5] = S / D;
    g[10] = S;
    g[15] = (r * r + a * a + 2 * a * a * r * s * s / S) * s * s;
    return g;
}
// ZAMO components (t, r, phi, -theta) of a BL contravariant vector (Krang's jac_zamo_u_bl_d).
inline M4 jac_zamo_u_bl_d(double a, double r, double th) {
    double s = std::sin(th), c = std::cos(th);
    double S = r * r + a * a * c * c, D = r * r - 2 * r + a * a;
    double A = (r * r + a * a) * (r * r + a * a) - a * a * D * s * s;
    double lapse = std::sqrt(S * D / A), om = 2 * a * r / A, varpi = std::sqrt(A / S) * s;
    M4 J{};
    J[0] = lapse;
    J[4 + 1] = std::sqrt(S / D);
    J[8 + 0] = -varpi * om; J[8 + 3] = varpi;
    J[12 + 2] = -std::sqrt(S);
    return J;
}
// Its inverse: BL contravariant components of a vector given in ZAMO components (jac_bl_u_zamo_d).
inline M4 jac_bl_u_zamo_d(double a, double r, double th) {
    double s = std::sin(th), c = std::cos(th);
    double S = r * r + a * a * c * c, D = r * r - 2 * r + a * a;
    double A = (r * r + a * a) * (r * r + a * a) - a * a * D * s * s;
    double lapse = std::sqrt(S * D / A), om = 2 * a * r / A, varpi = std::sqrt(A / S) * s;
    M4 J{};
    J[0] = 1.0 / lapse;
    J[4 + 1] = std::sqrt(D / S);
    J[8 + 3] = -1.0 / std::sqrt(S);
    J[12 + 0] = om / lapse; J[12 + 2] = 1.0 / varpi;
    return J;
}

inline double safe_sqrt(double x) { return x > 0 ? std::sqrt(x) : 0.0; }

// frames.jl:93-97
inline V4 momentum_bl_d(double a, double r, double th, double eta, double lam, bool nur, bool nuth) {
    double D = r * r - 2 * r + a * a;
    double pr = (nur ? 1.0 : -1.0) * safe_sqrt(r_potential(a, eta, lam, r)) / D;
    double pth = (nuth ? 1.0 : -1.0) * safe_sqrt(theta_potential(a, eta, lam, th));
    return {-1.0, pr, pth, lam};
}
// Krang's p_bl_d (used by the thin renderer, Splats.jl:123): the same momentum, square roots of the
// potentials clamped at zero.
inline V4 p_bl_d(double a, double r, double th, double eta, double lam, bool nur, bool nuth) {
    return momentum_bl_d(a, r, th, eta, lam, nur, nuth);
}

// frames.jl:31-41
inline M4 boost_zamo_to_fluid(double u1, double u2, double u3) {
    double u2s = u1 * u1 + u2 * u2 + u3 * u3;
    double g = std::sqrt(1 + u2s), q = 1.0 / (g + 1);
    return {g, -u1, -u2, -u3,
            -u1, 1 + u1 * u1 * q, u1 * u2 * q, u1 * u3 * q,
            -u2, u1 * u2 * q, 1 + u2 * u2 * q, u2 * u3 * q,
            -u3, u1 * u3 * q, u2 * u3 * q, 1 + u3 * u3 * q};
}

struct Frame { double g, cosB, chi; };

// frames.jl:108-128
inline Frame local_frame(double a, double r, double th, double eta, double lam, bool nur, bool nuth,
                         double alpha, double beta, double thetao, const double u[3], const double B[3]) {
    V4 pd = momentum_bl_d(a, r, th, eta, lam, nur, nuth);
    V4 pu = mv(metric_uu(a, r, th), pd);
    V4 pz = mv(jac_zamo_u_bl_d(a, r, th), pu);
    M4 L = boost_zamo_to_fluid(u[0], u[1], u[2]);
    V4 pf = mv(L, pz);
    double g = 1.0 / pf[0];
    double k[3] = {pf[1] * g, pf[2] * g, pf[3] * g};
    double Bn = std::sqrt(B[0] * B[0] + B[1] * B[1] + B[2] * B[2]);
    double Bh[3] = {0, 0, 1};
    if (Bn > 0) { Bh[0] = B[0] / Bn; Bh[1] = B[1] / Bn; Bh[2] = B[2] / Bn; }
    double cosB = k[0] * Bh[0] + k[1] * Bh[1] + k[2] * Bh[2];
    double f[3] = {k[1] * Bh[2] - k[2] * Bh[1], k[2] * Bh[0] - k[0] * Bh[2], k[0] * Bh[1] - k[1] * Bh[0]};
    double fn = std::sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
    if (!(fn > 0)) return {g, cosB, 0.0};
    V4 ff = {0.0, f[0] / fn, f[1] / fn, f[2] / fn};
    V4 fz = mv(boost_zamo_to_fluid(-u[0], -u[1], -u[2]), ff);
    V4 fbl = mv(jac_bl_u_zamo_d(a, r, th), fz);
    // walker_penrose (frames.jl:62-70)
    double sth = std::sin(th), cth = std::cos(th);
    double A = pu[0] * fbl[1] - pu[1] * fbl[0] + a * sth * sth * (pu[1] * fbl[3] - pu[3] * fbl[1]);
    double Bw = ((r * r + a * a) * (pu[3] * fbl[2] - pu[2] * fbl[3]) - a * (pu[0] * fbl[2] - pu[2] * fbl[0])) * sth;
    double k1 = A * r - Bw * a * cth, k2 = -(A * a * cth + Bw * r);
    // screen_direction (frames.jl:78-81)
    double mu = -(alpha + a * std::sin(thetao));
    double ea = beta * k2 - mu * k1, eb = beta * k1 + mu * k2;
    return {g, cosB, std::atan2(-ea, eb)};
}

// ---- step.jl ----------------------------------------------------------------------------------

// M_n(a) = int_0^1 t^n e^{-a t} dt, n = 0..9: for |a| < 1 the series sum_m (-a)^m/(m! (n+m+1)),
// 24 terms (coefficients generated from the formula); otherwise the upward recurrence
// M_n = (n M_{n-1} - e^{-a})/a (step.jl:239-268).
struct MomentTable {
    double c[10][24];
    MomentTable() {
        for (int n = 0; n < 10; ++n) {
            double fact = 1.0;
            for (int m = 0; m < 24; ++m) {
                if (m > 0) fact *= m;
                c[n][m] = ((m % 2) ? -1.0 : 1.0) / (fact * (n + m + 1));
            }
        }
    }
};
inline const MomentTable& moment_table() { static MomentTable t; return t; }
inline std::array<double, 10> moments(double a) {
    std::array<double, 10> M{};
    if (std::fabs(a) < 1) {
        const MomentTable& T = moment_table();
        for (int n = 0; n < 10; ++n) {
            double s = T.c[n][23];
            for (int m = 22; m >= 0; --m) s = std::fma(a, s, T.c[n][m]);
            M[n] = s;
        }
    } else {
        double e = std::exp(-a);
        M[0] = (1 - e) / a;
        for (int n = 1; n < 10; ++n) M[n] = (n * M[n - 1] - e) / a;
    }
    return M;
}
// step.jl:179-185
inline double phi_fn(double a) {
    if (std::fabs(a) < 1) return moments(a)[0];
    return -std::expm1(-a) / a;
}
inline double moment1(double a) { return moments(a)[1]; }
inline double versin(double b) { double s = std::sin(b / 2); return 2 * s * s; }
inline double sinhc_excess(double b) {
    if (std::fabs(b) < 0.1) { double b2 = b * b; return b2 / 6 * (1 + b2 / 20 * (1 + b2 / 42 * (1 + b2 / 72 * (1 + b2 / 110)))); }
    return std::sinh(b) / b - 1;
}
inline double sinc_deficit(double b) {
    if (std::fabs(b) < 0.1) { double b2 = b * b; return b2 / 6 * (1 - b2 / 20 * (1 - b2 / 42 * (1 - b2 / 72 * (1 - b2 / 110)))); }
    return 1 - std::sin(b) / b;
}
inline double sinhc(double b) { return std::fabs(b) < 0.1 ? 1 + sinhc_excess(b) : std::sinh(b) / b; }
inline double sinc_fn(double b) { return std::fabs(b) < 0.1 ? 1 - sinc_deficit(b) : std::sin(b) / b; }
// step.jl:226-236
inline void damped_hyperbolics(double a, double b, double& ecosh, double& esinhb, double& ecoshm1) {
    if (b < 1) {
        double e = std::exp(-a);
        double sh = std::sinh(b / 2);
        ecosh = e * std::cosh(b); esinhb = e * sinhc(b); ecoshm1 = e * 2 * sh * sh;
    } else {
        double em = std::exp(-(a - b)), ep = std::exp(-(a + b)), e = std::exp(-a);
        ecosh = (em + ep) / 2; esinhb = (em - ep) / (2 * b); ecoshm1 = (em - 2 * e + ep) / 2;
    }
}
// step.jl:273-331
inline double int_coshm1(double a, double b) {
    if (b < 0.1) { auto M = moments(a); double b2 = b * b; return b2 * (M[2] / 2 + b2 * (M[4] / 24 + b2 * (M[6] / 720 + b2 * M[8] / 40320))); }
    return (phi_fn(a - b) + phi_fn(a + b)) / 2 - phi_fn(a);
}
inline double int_versin_series(double a, double b) { auto M = moments(a); double b2 = b * b; return b2 * (M[2] / 2 - b2 * (M[4] / 24 - b2 * (M[6] / 720 - b2 * M[8] / 40320))); }
inline double int_cos_closed(double a, double b) { double s = std::sin(b), c = std::cos(b); return (a - std::exp(-a) * (a * c - b * s)) / (a * a + b * b); }
inline double int_sinc_deficit_series(double a, double b) { auto M = moments(a); double b2 = b * b; return b2 * (M[3] / 6 - b2 * (M[5] / 120 - b2 * (M[7] / 5040 - b2 * M[9] / 362880))); }
inline double int_sinc_closed(double a, double b) { double s = std::sin(b), c = std::cos(b); return (1 - std::exp(-a) * (a * s / b + c)) / (a * a + b * b); }
inline double int_versin(double a, double b) { return b < 0.1 ? int_versin_series(a, b) : phi_fn(a) - int_cos_closed(a, b); }
inline double int_cos(double a, double b) { return b < 0.1 ? phi_fn(a) - int_versin_series(a, b) : int_cos_closed(a, b); }
inline double int_sinc(double a, double b) { return b < 0.1 ? moment1(a) - int_sinc_deficit_series(a, b) : int_sinc_closed(a, b); }
inline double int_sinhc_excess(double a, double b) {
    if (b < 0.1) { auto M = moments(a); double b2 = b * b; return b2 * (M[3] / 6 + b2 * (M[5] / 120 + b2 * (M[7] / 5040 + b2 * M[9] / 362880))); }
    return (phi_fn(a - b) - phi_fn(a + b)) / (2 * b) - moment1(a);
}

inline M4 eye4() { return {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1}; }
inline M4 lin(double c0, const M4& A, double c1, const M4& B) { M4 C{}; for (int i = 0; i < 16; ++i) C[i] = c0 * A[i] + c1 * B[i]; return C; }

// step.jl:64-124 (on the rescaled coefficients)
inline void step_operator_scaled(const V4& al, const double rh[3], double D, M4& O, M4& Ej) {
    double aI = al[0], aQ = al[1], aU = al[2], aV = al[3];
    double rQ = rh[0], rU = rh[1], rV = rh[2];
    double a2 = aQ * aQ + aU * aU + aV * aV;
    double r2 = rQ * rQ + rU * rU + rV * rV;
    double a = aI * D;
    M4 K1 = {0, aQ, aU, aV, aQ, 0, rV, -rU, aU, -rV, 0, rQ, aV, rU, -rQ, 0};
    M4 I = eye4();
    if ((a2 + r2) * D * D < 1e-200) {
        double e = std::exp(-a);
        O = lin(e, I, -e * D, K1);
        Ej = lin(D * phi_fn(a), I, -D * D * moment1(a), K1);
        return;
    }
    M4 K2 = mm(K1, K1), K3 = mm(K2, K1);
    double ar = aQ * rQ + aU * rU + aV * rV;
    double h = (a2 - r2) / 2;
    double root = safe_sqrt(h * h + ar * ar);
    double L1sq, L2sq;
    if (h >= 0) { L1sq = h + root; L2sq = L1sq > 0 ? ar * ar / L1sq : 0.0; }
    else { L2sq = root - h; L1sq = L2sq > 0 ? ar * ar / L2sq : 0.0; }
    double L1 = safe_sqrt(L1sq), L2 = safe_sqrt(L2sq);
    double b1 = L1 * D, b2 = L2 * D;
    double Th = L1sq + L2sq;
    if (Th * D * D * (1 + (a2 + r2) * D * D) < 1e-17) {
        double e = std::exp(-a);
        for (int i = 0; i < 16; ++i) O[i] = e * (I[i] - D * K1[i] + (D * D / 2) * K2[i] - (D * D * D / 6) * K3[i]);
        auto M = moments(a);
        for (int i = 0; i < 16; ++i) Ej[i] = D * (M[0] * I[i] - (D * M[1]) * K1[i] + (D * D * M[2] / 2) * K2[i] - (D * D * D * M[3] / 6) * K3[i]);
        return;
    }
    M4 M2, M3;
    for (int i = 0; i < 16; ++i) { M2[i] = (L1sq * K1[i] - K3[i]) / Th; M3[i] = (L2sq * K1[i] + K3[i]) / Th; }
    double ecosh, esinhb, ecoshm1;
    damped_hyperbolics(a, b1, ecosh, esinhb, ecoshm1);
    double e = std::exp(-a);
    double c0 = (L2sq * ecosh + L1sq * e * std::cos(b2)) / Th;
    double c2 = (ecoshm1 + e * versin(b2)) / Th;
    double so = D * esinhb, sn = D * e * sinc_fn(b2);
    for (int i = 0; i < 16; ++i) O[i] = c0 * I[i] + c2 * K2[i] - so * M3[i] - sn * M2[i];
    double Ich = D * (phi_fn(a) + int_coshm1(a, b1));
    double Ic = D * int_cos(a, b2);
    double Ish = D * D * (moment1(a) + int_sinhc_excess(a, b1));
    double Is = D * D * int_sinc(a, b2);
    double C0 = (L2sq * Ich + L1sq * Ic) / Th;
    double C2 = D * (int_coshm1(a, b1) + int_versin(a, b2)) / Th;
    for (int i = 0; i < 16; ++i) Ej[i] = C0 * I[i] + C2 * K2[i] - Ish * M3[i] - Is * M2[i];
}
// step.jl:45-54
inline void step_operator(const V4& al, const double rh[3], double D, M4& O, M4& Ej) {
    double s = pow2_below(D);
    V4 as = {al[0] * s, al[1] * s, al[2] * s, al[3] * s};
    double rs[3] = {rh[0] * s, rh[1] * s, rh[2] * s};
    step_operator_scaled(as, rs, D / s, O, Ej);
    for (int i = 0; i < 16; ++i) Ej[i] *= s;
}
// step.jl:27-30
inline void transfer_step(const V4& j, const V4& al, const double rh[3], double D, M4& O, V4& E) {
    M4 Ej;
    step_operator(al, rh, D, O, Ej);
    E = mv(Ej, j);
}

// ---- splats (Splats.jl, polarized.jl, populations.jl, trajectories.jl) -------------------------

// Splats.jl:72-78
inline void quaternion_rotation(double q1, double q2, double q3, double q4, double R[9]) {
    double n = std::sqrt(q1 * q1 + q2 * q2 + q3 * q3 + q4 * q4);
    double w = q1 / n, x = q2 / n, y = q3 / n, z = q4 / n;
    R[0] = 1 - 2 * (y * y + z * z); R[1] = 2 * (x * y - w * z); R[2] = 2 * (x * z + w * y);
    R[3] = 2 * (x * y + w * z); R[4] = 1 - 2 * (x * x + z * z); R[5] = 2 * (y * z - w * x);
    R[6] = 2 * (x * z - w * y); R[7] = 2 * (y * z + w * x); R[8] = 1 - 2 * (x * x + y * y);
}
// Splats.jl:58-69 (p = one column, nrows rows; the pattern rate is the last row)
inline void pattern_offset(const double* p, int nrows, double t, double x, double y, double z, double u[3]) {
    double ph = p[nrows - 1] * (t - p[10]);
    double s = std::sin(ph), c = std::cos(ph);
    double cx = p[0] * c - p[1] * s, cy = p[0] * s + p[1] * c;
    double d0 = x - cx, d1 = y - cy, d2 = z - p[2];
    double dr0 = d0 * c + d1 * s, dr1 = -d0 * s + d1 * c, dr2 = d2;
    double R[9];
    quaternion_rotation(p[6], p[7], p[8], p[9], R);
    u[0] = R[0] * dr0 + R[3] * dr1 + R[6] * dr2;   // R' * dr
    u[1] = R[1] * dr0 + R[4] * dr1 + R[7] * dr2;
    u[2] = R[2] * dr0 + R[5] * dr1 + R[8] * dr2;
}
// Splats.jl:86-93
inline double splat_emissivity(const double* p, int nrows, double t, double x, double y, double z) {
    double u[3];
    pattern_offset(p, nrows, t, x, y, z, u);
    double e0 = u[0] * std::exp(-p[3]), e1 = u[1] * std::exp(-p[4]), e2 = u[2] * std::exp(-p[5]);
    double q2 = e0 * e0 + e1 * e1 + e2 * e2;
    double tt = (t - p[10]) * std::exp(-p[11]);
    return std::exp(p[12] - (q2 + tt * tt) / 2);
}
// polarized.jl:22-29
inline double splat_weight(const double* p, int nrows, double t, double x, double y, double z) {
    double u[3];
    pattern_offset(p, nrows, t, x, y, z, u);
    double e0 = u[0] * std::exp(-p[3]), e1 = u[1] * std::exp(-p[4]), e2 = u[2] * std::exp(-p[5]);
    double q2 = e0 * e0 + e1 * e1 + e2 * e2;
    double tt = (t - p[10]) * std::exp(-p[11]);
    return std::exp(-(q2 + tt * tt) / 2);
}
// polarized.jl:96-97, 110-120
constexpr double WEIGHT_CUTOFF = 1e-6;
inline double support_radius2() { return -2.0 * std::log(WEIGHT_CUTOFF); }
inline bool outside_support(const double* p, int nrows, double t, double x, double y, double z) {
    double ph = p[nrows - 1] * (t - p[10]);
    double s = std::sin(ph), c = std::cos(ph);
    double cx = p[0] * c - p[1] * s, cy = p[0] * s + p[1] * c;
    double d2 = (x - cx) * (x - cx) + (y - cy) * (y - cy) + (z - p[2]) * (z - p[2]);
    double smax = std::max({p[3], p[4], p[5]});
    return d2 > support_radius2() * std::exp(2 * smax);
}

enum SplatKind { KIND_THIN14 = 0, KIND_THERMAL21 = 1, KIND_POWERLAW22 = 2, KIND_KAPPA22 = 3, KIND_KNOT21 = 4 };

struct SplatSet {
    int kind;
    int nrows;
    int nsplat;
    const double* params;   // column-major nrows x nsplat
    double gmax = 1e5;      // power-law gamma_max (populations.jl:40)
    const double* hyp = nullptr;     // kappa hypergeometric factors per splat
    const double* knots = nullptr;   // 3 x nknots x nsplat
    const double* knot_times = nullptr;
    int nknots = 0;
};

struct RayCtx { const Ray* R; };

// trajectories.jl:93-111
inline void knot_centre(const SplatSet& S, int i, double t, double c[3]) {
    const double* ts = S.knot_times;
    int n = S.nknots;
    const double* K = S.knots + size_t(3) * n * i;
    if (t <= ts[0]) { c[0] = K[0]; c[1] = K[1]; c[2] = K[2]; return; }
    if (t >= ts[n - 1]) { c[0] = K[3 * (n - 1)]; c[1] = K[3 * (n - 1) + 1]; c[2] = K[3 * (n - 1) + 2]; return; }
    int k = 0;
    while (k < n - 2 && ts[k + 1] <= t) ++k;
    double w = (t - ts[k]) / (ts[k + 1] - ts[k]);
    for (int d = 0; d < 3; ++d) c[d] = (1 - w) * K[3 * k + d] + w * K[3 * (k + 1) + d];
}

// polarized.jl:140-150 (fluid rows -> frame -> coefficients), with the population of the set
inline bool element(const SplatSet& S, int i, const Ray& R, const Sample& s, double t_obs, double nu, Coeffs& cf, Frame& fr) {
    const double* p = S.params + size_t(S.nrows) * i;
    double x, y, z;
    quasi_cartesian_kerr_schild(R.a, s.r, s.theta, s.phi, x, y, z);
    double t = t_obs - s.t;
    double G;
    if (S.kind == KIND_KNOT21) {
        double c[3];
        knot_centre(S, i, t, c);
        double d[3] = {x - c[0], y - c[1], z - c[2]};
        double Rm[9];
        quaternion_rotation(p[6], p[7], p[8], p[9], Rm);
        double u0 = Rm[0] * d[0] + Rm[3] * d[1] + Rm[6] * d[2];
        double u1 = Rm[1] * d[0] + Rm[4] * d[1] + Rm[7] * d[2];
        double u2 = Rm[2] * d[0] + Rm[5] * d[1] + Rm[8] * d[2];
        double e0 = u0 * std::exp(-p[3]), e1 = u1 * std::exp(-p[4]), e2 = u2 * std::exp(-p[5]);
        double tt = (t - p[10]) * std::exp(-p[11]);
        G = std::exp(-(e0 * e0 + e1 * e1 + e2 * e2 + tt * tt) / 2);
        if (!(G > WEIGHT_CUTOFF)) return false;
    } else {
        if (outside_support(p, S.nrows, t, x, y, z)) return false;
        G = splat_weight(p, S.nrows, t, x, y, z);
        if (!(G > WEIGHT_CUTOFF)) return false;
    }
    int off = (S.kind == KIND_THERMAL21 || S.kind == KIND_KNOT21) ? 13 : 15;   // first field row (0-based): logB
    double Bmag, thB, phB, u[3];
    if (S.kind == KIND_THERMAL21 || S.kind == KIND_KNOT21) { Bmag = std::exp(p[14]); thB = p[15]; phB = p[16]; u[0] = p[17]; u[1] = p[18]; u[2] = p[19]; }
    else { Bmag = std::exp(p[15]); thB = p[16]; phB = p[17]; u[0] = p[18]; u[1] = p[19]; u[2] = p[20]; }
    (void)off;
    double B[3] = {Bmag * std::sin(thB) * std::cos(phB), Bmag * std::sin(thB) * std::sin(phB), Bmag * std::cos(thB)};
    fr = local_frame(R.a, s.r, s.theta, R.eta, R.lam, s.nur, s.nutheta, R.alpha, R.beta, R.thetao, u, B);
    double nuf = nu / fr.g;
    double thb = std::acos(std::max(-1.0, std::min(1.0, fr.cosB)));
    double ne = std::exp(p[12]) * G;
    if (S.kind == KIND_THERMAL21 || S.kind == KIND_KNOT21) cf = thermal_synchrotron(ne, std::exp(p[13]), Bmag, nuf, thb);
    else if (S.kind == KIND_POWERLAW22) cf = powerlaw_synchrotron(ne, p[13], std::exp(p[14]), S.gmax, Bmag, nuf, thb);
    else cf = kappa_synchrotron(ne, p[13], std::exp(p[14]), Bmag, nuf, thb, S.hyp[i]);
    return true;
}

// transport.jl:265-270 + step.jl:407-413
inline bool screen_coefficients(const Coeffs& cf, const Frame& fr, double nu, V4& j, V4& al, double rh[3]) {
    if (!(cf.jI > 0 || cf.aI > 0 || cf.rQ != 0 || cf.rV != 0)) return false;
    Coeffs ci = invariants(cap_polarization(cf), nu / fr.g);
    double s2 = std::sin(2 * fr.chi), c2 = std::cos(2 * fr.chi);
    j = {ci.jI, ci.jQ * c2, ci.jQ * s2, ci.jV};
    al = {ci.aI, ci.aQ * c2, ci.aQ * s2, ci.aV};
    rh[0] = ci.rQ * c2; rh[1] = ci.rQ * s2; rh[2] = ci.rV;
    return true;
}

// step.jl:342-347
struct RadState { M4 P; V4 S; };
inline RadState rad_zero() { return {eye4(), {0, 0, 0, 0}}; }
inline void advance(RadState& st, const M4& O, const V4& E) {
    V4 PE = mv(st.P, E);
    for (int i = 0; i < 4; ++i) st.S[i] += PE[i];
    st.P = mm(st.P, O);
}
// step.jl:362-398
struct Winding { double zprev; int n; bool inside, crossed; };
inline Winding winding_zero() { return {std::numeric_limits<double>::quiet_NaN(), 0, false, false}; }
inline Winding wind(const Winding& w, double z, double h) {
    if (std::isnan(w.zprev)) return {z, w.n, std::fabs(z) < h, false};
    bool inside_now = std::fabs(z) < h;
    bool crossing = w.zprev * z < 0;
    int n = w.n; bool inside = w.inside, crossed = w.crossed;
    if (inside || inside_now) {
        crossed = crossed || crossing;
        if (inside && !inside_now) { if (crossed) n += 1; crossed = false; }
        else if (!inside && inside_now) { crossed = crossing; }
        inside = inside_now;
    } else if (crossing) {
        n += 1;
    }
    return {z, n, inside, crossed};
}

// Sum of the screen coefficients of every element of several sets (transport.jl:296-306, 306-316)
inline bool accumulate_elements(const std::vector<SplatSet>& sets, const Ray& R, const Sample& s, double t_obs, double nu,
                                V4& j4, V4& a4, double r3[3]) {
    j4 = {0, 0, 0, 0}; a4 = {0, 0, 0, 0}; r3[0] = r3[1] = r3[2] = 0;
    bool active = false;
    for (const SplatSet& S : sets)
        for (int i = 0; i < S.nsplat; ++i) {
            Coeffs cf; Frame fr;
            if (!element(S, i, R, s, t_obs, nu, cf, fr)) continue;
            V4 jj, aa; double rr[3];
            if (!screen_coefficients(cf, fr, nu, jj, aa, rr)) continue;
            for (int q = 0; q < 4; ++q) { j4[q] += jj[q]; a4[q] += aa[q]; }
            for (int q = 0; q < 3; ++q) r3[q] += rr[q];
            active = true;
        }
    return active;
}

// RadiativeTransport consumer (transport.jl:171-198) over any element sum: `accum(s, j4, a4, r3)`
// fills the summed screen coefficients of a sample and says whether any element is active there.
// nmax >= 0 selects the winding consumer.
struct PolarizedResult { double I, Q, U, V; };
template <class Accum>
inline PolarizedResult polarized_ray_model(const Ray& R, int N, int M, double nu, double L, int nmax, double slab, Accum&& accum,
                                           double* resid_t = nullptr, double* resid_phi = nullptr) {
    RadState st = rad_zero();
    Winding w = winding_zero();
    double rh = horizon(R.a);
    double dtau = mino_step(R.tau_total, N);
    march_ray(R, N, M, [&](int, const Sample& s) {
        if (!(s.ok && s.r > rh * (1 + 1e-3))) return;
        if (nmax >= 0) {
            w = wind(w, s.r * std::cos(s.theta), slab);
            if (w.n > nmax) return;
        }
        V4 j4, a4; double r3[3];
        if (!accum(s, j4, a4, r3)) return;
        double ct = std::cos(s.theta);
        double Sg = s.r * s.r + R.a * R.a * ct * ct;
        double D = L / nuhat(nu) * Sg * dtau;
        M4 O; V4 E;
        transfer_step(j4, a4, r3, D, O, E);
        advance(st, O, E);
    }, resid_t, resid_phi);
    double n3 = nuhat(nu) * nuhat(nu) * nuhat(nu);
    return {st.S[0] * n3, st.S[1] * n3, st.S[2] * n3, st.S[3] * n3};
}

// The splat sets of a scene as the model (polarized.jl:121-130, transport.jl:306-316).
inline PolarizedResult polarized_ray(const Ray& R, int N, int M, const std::vector<SplatSet>& sets, double t_obs, double nu, double L,
                                     int nmax, double slab, double* resid_t = nullptr, double* resid_phi = nullptr) {
    return polarized_ray_model(R, N, M, nu, L, nmax, slab, [&](const Sample& s, V4& j4, V4& a4, double r3[3]) {
        return accumulate_elements(sets, R, s, t_obs, nu, j4, a4, r3);
    }, resid_t, resid_phi);
}

// ---- ipole's RIAF as a one-element fluid model (test/riaf_model.jl) ----------------------------
// A thick disk with power-law density and temperature, a toroidal field of equipartition-like
// strength, Keplerian rotation outside the ISCO and the conserved-quantity plunge inside it, thermal
// synchrotron with Pandya emissivities (ipole's emission_type 1).
struct RIAF { double nth0, Te0, disk_h, pow_nth, pow_T, Ne_unit, Te_unit, eps, r_isco, rout; bool pandya; };

// riaf_model.jl:25-29 (Bardeen, Press & Teukolsky 1972, prograde)
inline double isco_radius(double a) {
    double z1 = 1 + std::cbrt(1 - a * a) * (std::cbrt(1 + a) + std::cbrt(1 - a));
    double z2 = std::sqrt(3 * a * a + z1 * z1);
    return 3 + z2 - std::copysign(std::sqrt((3 - z1) * (3 + z1 + 2 * z2)), a);
}
// riaf_model.jl:31-34 (ipole's model/riaf/example.par)
inline RIAF riaf_example(double a, bool pandya = true) {
    return {1.0, 1.0, 0.1, -1.1, -0.84, 3e7, 3e11, 0.1, isco_radius(a), 100.0, pandya};
}
inline double quad(const M4& g, const V4& x, const V4& y) {
    double s = 0;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) s += x[i] * g[4 * i + j] * y[j];
    return s;
}
// riaf_model.jl:38-93: the coefficients and the local frame of the RIAF at one sample; false where
// the model is empty (inside r_h + 0.1 or beyond rout).
inline bool riaf_element(const RIAF& m, const Ray& R, const Sample& s, double nu, Coeffs& cf, Frame& fr) {
    const double a = R.a, r = s.r, th = s.theta;
    const double rh = horizon(a);
    if (!(r > rh + 0.1 && r < m.rout)) return false;
    double sth = std::sin(th), cth = std::cos(th);
    double zc = r * cth, rc = r * sth;
    double n = m.nth0 * std::exp(-zc * zc / 2 / rc / rc / m.disk_h / m.disk_h) * std::pow(r, m.pow_nth) * m.Ne_unit;
    double Te = m.Te0 * std::pow(r, m.pow_T) * m.Te_unit * KBOL / (ME * CL * CL);
    double bmag = std::sqrt(8 * PI * m.eps * n * MP * CL * CL / 6 / r);
    if (bmag == 0) bmag = 1e-6;
    M4 gdd = metric_dd(a, r, th), guu = metric_uu(a, r, th);
    double om, ur;
    if (r < m.r_isco) {
        double wisco = 1 / (std::pow(m.r_isco, 1.5) + a);
        M4 gi = metric_dd(a, m.r_isco, th);
        V4 ui = {1.0, 0.0, 0.0, wisco};
        double nrm = std::sqrt(-quad(gi, ui, ui));
        for (double& x : ui) x /= nrm;
        V4 ud = mv(gi, ui);
        double e = ud[0], l = ud[3];
        double Kcon = guu[0] * e * e + 2 * guu[3] * e * l + guu[15] * l * l;
        double urk = -std::sqrt(std::max(0.0, -(1 + Kcon) / guu[5]));
        V4 ut = mv(guu, V4{e, urk, 0.0, l});
        om = ut[3] / ut[0];
        ur = ut[1];
    } else {
        om = 1 / (std::pow(r, 1.5) + a);
        ur = 0.0;
    }
    double K = gdd[0] + 2 * om * gdd[3] + om * om * gdd[15];
    double ut = std::sqrt(std::max(0.0, -(1 + ur * ur * gdd[5]) / K));
    V4 u = {ut, ur, 0.0, om * ut};
    // toroidal field projected orthogonal to u, normalised to bmag
    V4 Bc = {0.0, 0.0, 0.0, 1.0};
    double BdotU = quad(gdd, Bc, u);
    V4 b;
    for (int i = 0; i < 4; ++i) b[i] = Bc[i] + BdotU * u[i];
    double bn = bmag / std::sqrt(quad(gdd, b, b));
    for (double& x : b) x *= bn;
    // ZAMO velocity and the fluid-frame field
    M4 J = jac_zamo_u_bl_d(a, r, th);
    V4 uz = mv(J, u);
    double ut3[3] = {uz[1], uz[2], uz[3]};
    V4 bz = mv(boost_zamo_to_fluid(ut3[0], ut3[1], ut3[2]), mv(J, b));
    double Bf[3] = {bz[1], bz[2], bz[3]};
    fr = local_frame(a, r, th, R.eta, R.lam, s.nur, s.nutheta, R.alpha, R.beta, R.thetao, ut3, Bf);
    double nuf = nu / fr.g;
    double thB = std::acos(std::max(-1.0, std::min(1.0, fr.cosB)));
    cf = thermal_synchrotron(n, Te, bmag, nuf, thB, false, m.pandya);
    return true;
}

// The RIAF through the RadiativeTransport consumer (stokes_image of test/test_polarized.jl:54-61).
// `mirror_chi` negates the screen angle (a planted convention error for the tests: it must fail the
// comparison with ipole's images).
inline PolarizedResult riaf_ray(const Ray& R, int N, int M, const RIAF& m, double nu, double L, bool mirror_chi = false) {
    return polarized_ray_model(R, N, M, nu, L, -1, 0.0, [&](const Sample& s, V4& j4, V4& a4, double r3[3]) {
        Coeffs cf; Frame fr;
        if (!riaf_element(m, R, s, nu, cf, fr)) return false;
        if (mirror_chi) fr.chi = -fr.chi;
        return screen_coefficients(cf, fr, nu, j4, a4, r3);
    });
}

// ThinRenderer (Splats.jl:113-128); params THIN14, column-major
inline double thin_ray(const Ray& R, int N, int M, const double* params, int nsplat, double t_obs,
                       double* resid_t = nullptr, double* resid_phi = nullptr) {
    double acc = 0.0;
    double rh = horizon(R.a);
    double dtau = mino_step(R.tau_total, N);
    march_ray(R, N, M, [&](int, const Sample& s) {
        if (!(s.ok && rh * (1 + 1e-3) < s.r && s.r < 1e3)) return;
        double x, y, z;
        quasi_cartesian_kerr_schild(R.a, s.r, s.theta, s.phi, x, y, z);
        double t = t_obs - s.t;
        double jt = 0.0;
        for (int i = 0; i < nsplat; ++i) jt += splat_emissivity(params + 14 * size_t(i), 14, t, x, y, z);
        V4 pbl = p_bl_d(R.a, s.r, s.theta, R.eta, R.lam, s.nur, s.nutheta);
        V4 pz = mv(jac_zamo_u_bl_d(R.a, s.r, s.theta), mv(metric_uu(R.a, s.r, s.theta), pbl));
        double g = 1.0 / pz[0];
        double ct = std::cos(s.theta);
        double Sg = s.r * s.r + R.a * R.a * ct * ct;
        acc += g * g * jt * Sg * dtau;
    }, resid_t, resid_phi);
    return acc;
}

}  // namespace kso
