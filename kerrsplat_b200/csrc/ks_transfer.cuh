// ks_transfer.cuh -- the transport consumers in precision T: splat tables, synchrotron coefficients,
// local frames and the exact constant-coefficient 4x4 Stokes step.
//
// Restates src/Transfer/{coefficients,kappa,frames,step,transport}.jl and
// src/Splats/{Splats,polarized,populations,trajectories}.jl (cited per function). Everything that
// depends only on a splat's parameters (exp of the scales, the quaternion rotation, the field
// vector, Bessel ratios of 1/Theta_e, Gamma-function products) is evaluated once per splat in FP64
// by the splat-table kernel and staged in shared memory; the per-sample work keeps only what
// depends on the sample. The formulas are written in the scalar type T so that FP32 runs them
// without leaving FP32's range (the reference's own constraint, coefficients.jl:147-152).
#pragma once
#include "ks_dual.cuh"
#include "ks_march.cuh"

namespace ks {

// constants.jl:3-12 (ipole / symphony cgs values) and coefficients.jl:299-303
constexpr double kME = 9.1093826e-28, kCL = 2.99792458e10, kEE = 4.80320680e-10, kHPL = 6.6260693e-27;
constexpr double kNU0 = 1e11;
constexpr double kPLANCK0 = 2.0 * kHPL * kNU0 * kNU0 * kNU0 / (kCL * kCL);
constexpr double kWEIGHT_CUTOFF = 1e-6;

// ---- splat table (FP64, per splat) ----------------------------------------------------------------
enum SplatTab {
    ST_CX, ST_CY, ST_CZ, ST_T0, ST_OMEGA, ST_ES1, ST_ES2, ST_ES3,
    ST_R0, ST_R1, ST_R2, ST_R3, ST_R4, ST_R5, ST_R6, ST_R7, ST_R8,
    ST_INVW, ST_SUPP, ST_NE, ST_LOGA,
    ST_TE, ST_F0, ST_KR,
    ST_BMAG, ST_BHX, ST_BHY, ST_BHZ, ST_U1, ST_U2, ST_U3, ST_BZERO,
    ST_P, ST_GMIN, ST_GMAX, ST_GSPAN, ST_GAMJ, ST_GAMA,
    ST_KAP, ST_W, ST_HYP, ST_G43, ST_G2, ST_GQ, ST_GP, ST_GK2, ST_KB,
    ST_KIND, ST_RHO,
    ST_KOFF, ST_NK,           // knot splats: offset of the splat's knot record in the knot array, knot count
    ST_COUNT
};

// ---- small helpers --------------------------------------------------------------------------------
template <class T> __device__ __forceinline__ T sq(T x) { return x * x; }

// 2^floor(log2 v) (step.jl:57-62), exact
__device__ __forceinline__ double pow2_below(double v) {
    if (!(isfinite(v) && v > 0)) return 1.0;
    int e; frexp(v, &e);
    return ldexp(1.0, e - 1);
}
__device__ __forceinline__ float pow2_below(float v) {
    if (!(isfinite(v) && v > 0)) return 1.0f;
    int e; frexpf(v, &e);
    return ldexpf(1.0f, e - 1);
}

// Transcendentals of the coefficient fits: the hardware approximations in FP32 (relative errors of a
// few 1e-6 at the arguments these fits take, inside the mixed path's 1e-4 budget), the correctly
// rounded library functions in FP64.
__device__ __forceinline__ float fpow(float x, float y) { return __powf(x, y); }
__device__ __forceinline__ double fpow(double x, double y) { return pow(x, y); }
__device__ __forceinline__ float fexp(float x) { return __expf(x); }
__device__ __forceinline__ double fexp(double x) { return exp(x); }
__device__ __forceinline__ float flog(float x) { return __logf(x); }
__device__ __forceinline__ double flog(double x) { return log(x); }
// Sine and cosine of a phase. FP32: the argument is reduced by 2 pi split in two floats (Cody & Waite
// 1980; 2 pi = 6.2831854820251465 - 1.7484555314695172e-7 to FP32's precision twice) and the hardware
// approximations run on [-pi, pi] (absolute error ~4e-7, below the FP32 rounding of the phases these
// take, a few to a thousand radians). FP64 and dual numbers: the library functions.
__device__ __forceinline__ float freduce(float x) {
    const float k = rintf(x * 0.15915494309189535f);
    const float r = fmaf(-k, 6.2831854820251465f, x);
    return fmaf(-k, -1.7484555314695172e-7f, r);
}
__device__ __forceinline__ void fsincos(float x, float& s, float& c) { __sincosf(freduce(x), &s, &c); }
__device__ __forceinline__ float fcos(float x) { return __cosf(freduce(x)); }
template <class T> __device__ __forceinline__ void fsincos(const T& x, T& s, T& c) { s = sin(x); c = cos(x); }
template <class T> __device__ __forceinline__ T fcos(const T& x) { return cos(x); }
// FP32 duals: the value by the reduced hardware pair, the partials by the chain rule
template <int N> __device__ __forceinline__ void fsincos(const Dual<float, N>& x, Dual<float, N>& s, Dual<float, N>& c) {
    float sv, cv;
    fsincos(x.v, sv, cv);
    s = dchain(x, sv, cv);
    c = dchain(x, cv, -sv);
}
template <int N> __device__ __forceinline__ Dual<float, N> fcos(const Dual<float, N>& x) {
    float sv, cv;
    fsincos(x.v, sv, cv);
    return dchain(x, cv, -sv);
}
// the same for dual numbers (the adjoint's forward-mode derivatives)
template <class T, int N> __device__ __forceinline__ Dual<T, N> fexp(const Dual<T, N>& x) { T e = fexp(x.v); return dchain(x, e, e); }
template <class T, int N> __device__ __forceinline__ Dual<T, N> flog(const Dual<T, N>& x) { return dchain(x, flog(x.v), T(1) / x.v); }
template <class T, int N>
__device__ __forceinline__ Dual<T, N> fpow(const Dual<T, N>& x, const Dual<T, N>& y) {
    Dual<T, N> r;
    r.v = fpow(x.v, y.v);
    bool ydep = false;
#pragma unroll
    for (int i = 0; i < N; ++i) ydep = ydep || (y.d[i] != T(0));
    const T dx = x.v != T(0) ? y.v * r.v / x.v : (y.v == T(1) ? T(1) : T(0));
    const T dy = ydep ? r.v * flog(x.v) : T(0);
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = dx * x.d[i] + (ydep ? dy * y.d[i] : T(0));
    return r;
}
// a power-of-two rescaling is exact: constant in the partials
template <class T, int N> __device__ __forceinline__ Dual<T, N> pow2_below(const Dual<T, N>& v) { return Dual<T, N>(pow2_below(v.v)); }

// ---- coefficients.jl ------------------------------------------------------------------------------
template <class T>
struct Coef { T jI, jQ, jV, aI, aQ, aV, rQ, rV; };

template <class T>
__device__ __forceinline__ T planck(T nu, T Te) {
    T x = T(kHPL) * nu / (T(kME) * T(kCL) * T(kCL) * Te);
    T nh = nu / T(kNU0);
    T pref = T(kPLANCK0) * nh * nh * nh;
    if (x < T(2e-3)) return pref / (x / T(24) * (T(24) + x * (T(12) + x * (T(4) + x))));
    if constexpr (is_f32<T>) return pref / expm1(x);   // no cancellation in FP32
    return pref / (exp(x) - T(1));
}

// coefficients.jl:101-145 with the Bessel ratios of the splat table (f0 = K0/K2, kr = K1/K2, both 1
// where K2 underflows)
template <class T>
__device__ __forceinline__ Coef<T> thermal_cs(T ne, T Te, T f0, T kr, T B, T nu, T st, T ct) {
    const T PI = kpi<T>();
    T w0 = T(kEE) * B / (T(kME) * T(kCL));
    T wp2 = T(4) * PI * ne * T(kEE) * T(kEE) / T(kME);
    T w = T(2) * PI * nu;
    T w0w = w0 / w, wp2w2 = wp2 / (w * w);
    if (!(st > T(0))) {
        T rV0 = w / T(kCL) * (wp2w2 * w0w * f0 * ct);
        return {T(0), T(0), T(0), T(0), T(0), T(0), T(0), rV0};
    }
    T x = Te * sqrt(T(1.4142135623730951) * st * (T(1e3) * w0w));
    T sw;   // 0.5 + 0.5 tanh((ln x - ln 120) / 0.1)
    if constexpr (is_f32<T>) {
        // = x^20 / (x^20 + 120^20): the same function without log and tanh, as p^20 / (1 + p^20) with
        // p = x / 120 below 120 and 1 / (1 + q^20) with q = 120 / x above (no overflow, so duals stay finite)
        const bool lo = x < T(120);
        const T q = lo ? x / T(120) : T(120) / x;
        const T q2 = q * q, q4 = q2 * q2, q5 = q4 * q, q10 = q5 * q5, q20 = q10 * q10;
        sw = lo ? q20 / (T(1) + q20) : T(1) / (T(1) + q20);
    } else {
        sw = T(0.5) + T(0.5) * tanh((flog(x) - T(4.787491742782046 /* ln 120 */)) / T(0.1));
    }
    T extraterm = (T(0.011) * fexp(-x / T(47.2)) - T(7.9370052598409974e-01 /* 2^(-1/3) */) / T(67.44733739010397 /* 3^(23/6) */) * PI * T(1e4) * fpow(x + T(1e-16), T(-8.0 / 3))) *
                  sw;
    T jffunc = T(2.011) * fexp(-fpow(x, T(1.035)) / T(4.7)) - fcos(x / T(2)) * fexp(-fpow(x, T(1.2)) / T(2.73)) - T(0.011) * fexp(-x / T(47.2)) + extraterm;
    T eps11m22 = jffunc * wp2w2 * w0w * w0w * (kr + T(6) * Te) * st * st;
    T rQ = w / (T(2) * T(kCL)) * eps11m22;
    T ff = f0 * (T(1) - T(0.11) * flog(T(1) + T(0.035) * x));
    T rV = w / T(kCL) * (wp2w2 * w0w * ff * ct);
    T nus = T(3) * T(kEE) * B * st / (T(4) * PI * T(kME) * T(kCL)) * Te * Te + T(1);
    T xs = nu / nus;
    T c13 = fpow(xs, T(-1.0 / 3)), c23 = c13 * c13;
    T e13 = fexp(T(-1.8899) / c13);     // fexp(-1.8899 x^(1/3))
    T pref = ne * T(kEE) * T(kEE) * nu / (T(2) * T(1.7320508075688772) * T(kCL) * Te * Te);
    T jI = pref * T(2.5651) * (T(1) + T(1.92) * c13 + T(0.9977) * c23) * e13;
    T jQ = pref * T(2.5651) * (T(1) + T(0.93193) * c13 + T(0.499873) * c23) * e13;
    T jV = T(2) * ne * T(kEE) * T(kEE) * nu * ct / st / (T(3) * T(1.7320508075688772) * T(kCL) * Te * Te * Te) *
           ((T(1.81384) / xs + T(3.42319) * c23 + T(0.0292545) * fpow(xs, T(-0.5)) + T(2.03773) * c13) * e13);
    T Bn = planck(nu, Te);
    T invB = Bn > T(0) ? T(1) / Bn : T(0);
    return {jI, jQ, jV, jI * invB, jQ * invB, jV * invB, rQ, rV};
}

// coefficients.jl:147-169: the Pandya et al. (2016) thermal emissivities (ipole's emission_type 1) at
// the pitch angle whose sine and cosine are st, ct; sin(theta - 28/25) by the angle-difference rule.
template <class T>
__device__ __forceinline__ void pandya_emissivities(T ne, T Te, T B, T nu, T st, T ct, T& jI, T& jQ, T& jV) {
    const T PI = kpi<T>();
    T nuc = T(kEE) * B / (T(2) * PI * T(kME) * T(kCL));
    T nus = T(2.0 / 9.0) * nuc * st * Te * Te;
    T X = nu / nus;
    T pref = ne * T(kEE) * T(kEE) * nuc / T(kCL);
    T term1 = T(1.4142135623730951) * PI / T(27) * st;
    T x13 = fpow(X, T(1.0 / 3)), x16 = fpow(X, T(1.0 / 6)), x12 = sqrt(X);
    const T c1112 = T(1.8877486253633868);   // 2^(11/12)
    T ex = fexp(-x13);
    T bi = x12 + c1112 * x16;
    jI = pref * term1 * bi * bi * ex;
    T te = fpow(Te, T(24.0 / 25));
    T t2 = (T(7) * te + T(35)) / (T(10) * te + T(75));
    T bq = x12 + t2 * c1112 * x16;
    jQ = pref * term1 * bq * bq * ex;
    T s28 = st * T(0.4356824462767121 /* cos(28/25) */) - ct * T(0.9001004421765051 /* sin(28/25) */);
    T tv1 = (T(37) - T(87) * s28) / (T(100) * (Te + T(1)));
    T tv2 = fpow(T(1) + (fpow(Te, T(3.0 / 5)) / T(25) + T(7.0 / 10)) * fpow(X, T(9.0 / 25)), T(5.0 / 3));
    jV = pref * tv1 * tv2 * ex;
}

// coefficients.jl:208-256 (Pandya+ 2016 power-law fits, Jones & O'Dell rotativities); gamj, gama are
// the splat's Gamma-function products, gspan = gmin^(1-p) - gmax^(1-p)
template <class T>
__device__ __forceinline__ Coef<T> powerlaw_cs(T ne, T p, T gmin, T gspan, T gamj, T gama, T B, T nu, T st, T ct) {
    // the fits divide by sin(theta) and raise it to negative powers: a field along the ray (a pitch
    // angle that rounds to 0 or pi, common in FP32) is evaluated 1e-6 from the axis
    st = fmax(st, T(1e-6));
    const T PI = kpi<T>();
    T nc = T(kEE) * B / (T(2) * PI * T(kME) * T(kCL));
    T pref = ne * T(kEE) * T(kEE) * nc / T(kCL);
    T xx = nu / (nc * st);
    T jI = pref * (fpow(T(3), p / T(2)) * (p - T(1)) * st) / (T(2) * (p + T(1)) * gspan) * gamj * fpow(xx, -(p - T(1)) / T(2));
    T jQ = (p + T(1)) / (p + T(7.0 / 3)) * jI;
    T jV = T(171.0 / 250) * fpow(p, T(49.0 / 100)) * ct / st * fpow(nu / (T(3) * nc * st), T(-0.5)) * jI;
    T apref = ne * T(kEE) * T(kEE) / (nu * T(kME) * T(kCL));
    T aI = apref * fpow(T(3), (p + T(1)) / T(2)) * (p - T(1)) / (T(4) * gspan) * gama * fpow(xx, -(p + T(2)) / T(2));
    T aQ = aI * fpow(T(17.0 / 500) * p - T(43.0 / 1250), T(43.0 / 500));
    T term6 = fpow(T(31.0 / 10) * fpow(st, T(-48.0 / 25)) - T(31.0 / 10), T(64.0 / 125));
    T sg = ct > T(0) ? T(1) : (ct < T(0) ? T(-1) : T(0));
    T aV = aI * fpow(T(71.0 / 100) * p + T(22.0 / 625), T(197.0 / 500)) * term6 * fpow(xx, T(-0.5)) * sg;
    // rotativities
    T nB = T(kEE) * B * st / (T(2) * PI * T(kME) * T(kCL));
    T rperp = ne * T(kEE) * T(kEE) * (p - T(1)) / (T(kME) * T(kCL) * nB * gspan);
    T nmin = gmin * gmin * nB;
    T rQ = -rperp * fpow(nB / nu, T(3)) * fpow(gmin, T(2) - p) * (T(1) - fpow(nmin / nu, p / T(2) - T(1))) / (p / T(2) - T(1));
    T rV = T(2) * (p + T(2)) / (p + T(1)) * rperp * sq(nB / nu) * fpow(gmin, -(p + T(1))) * flog(gmin) * ct / st;
    return {jI, jQ, jV, aI, aQ, aV, rQ, rV};
}

// kappa.jl:158-203 (Marszewski+ 2021 rotativity fits)
template <class T>
__device__ __forceinline__ T kappa_rhoQ_fit(int i, T w, T X) {
    T sw = sqrt(w), e5 = fexp(T(-5) * w), x84 = fpow(X, T(0.84));
    if (i == 1) return (T(17) * w - T(3) * sw + T(7) * sw * e5) * (T(1) - fexp(-x84 / T(30)) - sin(X / T(10)) * fexp(T(-3) * fpow(X, T(0.471)) / T(2)));
    if (i == 2) return (T(46) * w / T(3) - T(5) * sw / T(3) + T(17) * sw / T(3) * e5) * (T(1) - fexp(-x84 / T(18)) - sin(X / T(6)) * fexp(T(-7) * fpow(X, T(0.5)) / T(4)));
    if (i == 3) return (T(14) * w - T(13) * sw / T(8) + T(9) * sw / T(2) * e5) * (T(1) - fexp(-x84 / T(12)) - sin(X / T(4)) * fexp(T(-2) * fpow(X, T(0.525))));
    return (T(25) * w / T(2) - sw + T(5) * sw * e5) * (T(1) - fexp(-x84 / T(8)) - sin(T(3) * X / T(8)) * fexp(T(-9) * fpow(X, T(0.541)) / T(4)));
}
template <class T>
__device__ __forceinline__ T kappa_rhoV_fit(int i, T w, T X) {
    T xm = fpow(X, T(-0.5));
    if (i == 1) return (w * w + T(2) * w + T(1)) / (T(25) * w * w / T(8) + T(4) * w + T(1)) * (T(1) - T(0.17) * flog(T(1) + T(0.447) * xm));
    if (i == 2) return (w * w + T(54) * w + T(50)) / (T(30) * w * w / T(11) + T(134) * w + T(50)) * (T(1) - T(0.17) * flog(T(1) + T(0.391) * xm));
    if (i == 3) return (w * w + T(43) * w + T(38)) / (T(7) * w * w / T(3) + T(185) * w / T(2) + T(38)) * (T(1) - T(0.17) * flog(T(1) + T(0.348) * xm));
    return (w + T(13.0 / 14)) / (T(2) * w + T(13.0 / 14)) * (T(1) - T(0.17) * flog(T(1) + T(0.313) * xm));
}

// kappa.jl:109-155; g43 = Gamma(k - 4/3), g2 = Gamma(k - 2), gq = Gamma(k/4 - 1/3), gp = Gamma(k/4 + 4/3),
// gk2 = Gamma(2 + k/2), kb = K0/(K2 + 1e-40) at 1/w (per splat)
template <class T>
__device__ __forceinline__ Coef<T> kappa_cs(T ne, T kap, T w, T hyp, T g43, T g2, T gq, T gp, T gk2, T kb, T B, T nu, T st, T ct) {
    st = fmax(st, T(1e-6));   // as powerlaw: a field along the ray is evaluated 1e-6 from the axis
    const T PI = kpi<T>();
    const T small = T(1e-40);  // FP32: subnormal-flushes to 0; the guard below then reads |N_high| < 0
    T nc = T(kEE) * B / (T(2) * PI * T(kME) * T(kCL));
    T nw = (w * kap) * (w * kap) * nc * st;
    T X = nu / nw;
    T pref = ne * T(kEE) * T(kEE) * nc * st / T(kCL);
    T c373 = T(12.980246132766677);  // 3^(7/3)
    T NlowI = T(4) * PI * g43 / (c373 * g2);
    T hk = T(0.25) * fpow(T(3), (kap - T(1)) / T(2)) * (kap - T(2)) * (kap - T(1)) * gq * gp;
    T NhighI = hk + small;
    T xI = T(3) * fpow(kap, T(-1.5));
    T X13 = fpow(X, T(1.0 / 3));
    T jI = pref * NlowI * X13 * fpow(T(1) + fpow(X, xI * (T(3) * kap - T(4)) / T(6)) * fpow(NlowI / NhighI, xI), T(-1) / xI);
    T NlowQ = T(-0.5) * T(4) * PI * g43 / (c373 * g2);
    T NhighQ = -(T(0.64) + kap / T(50)) * hk + small;
    T xQ = T(3.7) * fpow(kap, T(-1.6));
    T jQ = -(pref * NlowQ * X13 * fpow(T(1) + fpow(X, xQ * (T(3) * kap - T(4)) / T(6)) * fpow(NlowQ / NhighQ, xQ), T(-1) / xQ));
    T NlowV = -T(0.5625) * fpow(fpow(st, T(-12.0 / 5)) - T(1), T(12.0 / 25)) * (fpow(kap, T(-66.0 / 125)) / w) * fpow(X, T(-7.0 / 20)) * T(4) * PI * g43 / (c373 * g2);
    T NhighV = -T(0.765625) * fpow(fpow(st, T(-2.5)) - T(1), T(11.0 / 25)) * (fpow(kap, T(-11.0 / 25)) / w) * fpow(X, T(-0.5)) * hk - small;
    T xV = T(3) * fpow(kap, T(-1.5));
    T sg = ct > T(0) ? T(1) : (ct < T(0) ? T(-1) : T(0));
    const T small2 = is_f32<T> ? T(0) : T(1e-80);   // small^2 (zero in FP32)
    T jV = fabs(NhighV) < small2 ? T(0)
         : -(pref * NlowV * X13 * fpow(T(1) + fpow(X, xV * (T(3) * kap - T(4)) / T(6)) * fpow(NlowV / NhighV, xV), T(-1) / xV)) * sg;
    T apref = ne * T(kEE) / (B * st);
    T g53 = T(0.9027452929509336);  // Gamma(5/3)
    T ck = (kap - T(2)) * (kap - T(1)) * kap;
    T c16 = T(1.2009369551760027);  // 3^(1/6)
    T base = c16 * T(10.0 / 41) * T(4) * PI * PI / fpow(w * kap, T(16.0 / 3) - kap) * ck / (T(3) * kap - T(1)) * g53 * hyp;
    T hiA = T(2) * fpow(PI, T(2.5)) / T(3) * ck / fpow(w * kap, T(5)) * (T(2) * gk2 / (T(2) + kap) - T(1));
    T NlowA = base;
    T NhighA = hiA * (fpow(T(3) / kap, T(19.0 / 4)) + T(3.0 / 5)) + small;
    T xA = fpow(T(-7.0 / 4) + T(8) * kap / T(5), T(-43.0 / 50));
    T X53 = fpow(X, T(-5.0 / 3));
    T aI = apref * NlowA * X53 * fpow(T(1) + fpow(X, xA * (T(3) * kap - T(1)) / T(6)) * fpow(NlowA / NhighA, xA), T(-1) / xA);
    T NlowQA = -T(25.0 / 48) * base;
    T NhighQA = -(T(441) * fpow(kap, T(-144.0 / 25)) + T(11.0 / 20)) * hiA + small;
    T xQA = T(1.4) * fpow(kap, T(-23.0 / 20));
    T aQ = -(apref * NlowQA * X53 * fpow(T(1) + fpow(X, xQA * (T(3) * kap - T(1)) / T(6)) * fpow(NlowQA / NhighQA, xQA), T(-1) / xQA));
    T NlowVA = -(T(77) / (T(100) * w)) * fpow(fpow(st, T(-114.0 / 50)) - T(1), T(223.0 / 500)) * fpow(X, T(-7.0 / 20)) * fpow(kap, T(-0.7)) * base;
    T NhighVA = -(T(14.3) * fpow(w, T(-116.0 / 125))) * fpow(fpow(st, T(-41.0 / 20)) - T(1), T(0.5)) *
                (T(169) * fpow(kap, T(-8)) + T(13.0 / 2500) * kap - T(263.0 / 5000) + T(47) / (T(200) * kap)) * fpow(X, T(-0.5)) * hiA + small;
    T xVA = T(1.22) * fpow(kap, T(-142.0 / 125)) + T(7.0 / 1000);
    T aV = -(apref * NlowVA * X53 * fpow(T(1) + fpow(X, xVA * (T(3) * kap - T(1)) / T(6)) * fpow(NlowVA / NhighVA, xVA), T(-1) / xVA)) * sg;
    // rotativities (kappa.jl:188-203)
    T Xr = nu / ((w * kap) * (w * kap) * nc * st);
    T kc = fmin(T(5), fmax(T(3.5), kap));
    int i = kc < T(4) ? 1 : (kc < T(4.5) ? 2 : 3);
    T klo = T(3.5) + T(i - 1) / T(2), f = (kc - klo) * T(2);
    T fQ = (T(1) - f) * kappa_rhoQ_fit(i, w, Xr) + f * kappa_rhoQ_fit(i + 1, w, Xr);
    T fV = (T(1) - f) * kappa_rhoV_fit(i, w, Xr) + f * kappa_rhoV_fit(i + 1, w, Xr);
    T rQ = -(ne * T(kEE) * T(kEE) * nc * nc * st * st) / (T(kME) * T(kCL) * nu * nu * nu) * fQ;
    T rV = T(2) * (ne * T(kEE) * T(kEE) * nc * ct) / (T(kME) * T(kCL) * nu * nu) * kb * fV;
    return {jI, jQ, jV, aI, aQ, aV, rQ, rV};
}

// The fits at the pitch angle th (the reference's signatures): its sine and cosine.
template <class T>
__device__ __forceinline__ Coef<T> thermal(T ne, T Te, T f0, T kr, T B, T nu, T th) { return thermal_cs(ne, Te, f0, kr, B, nu, sin(th), cos(th)); }
template <class T>
__device__ __forceinline__ Coef<T> powerlaw(T ne, T p, T gmin, T gspan, T gamj, T gama, T B, T nu, T th) {
    return powerlaw_cs(ne, p, gmin, gspan, gamj, gama, B, nu, sin(th), cos(th));
}
template <class T>
__device__ __forceinline__ Coef<T> kappa(T ne, T kap, T w, T hyp, T g43, T g2, T gq, T gp, T gk2, T kb, T B, T nu, T th) {
    return kappa_cs(ne, kap, w, hyp, g43, g2, gq, gp, gk2, kb, B, nu, sin(th), cos(th));
}
// The pitch angle's sine and cosine from its (clamped) cosine: sin(acos c) = sqrt((1 - c)(1 + c)).
template <class T>
__device__ __forceinline__ void pitch_sc(T cosB, T& st, T& ct) {
    ct = fmin(T(1), fmax(T(-1), cosB));
    const T s2 = (T(1) - ct) * (T(1) + ct);
    st = s2 > T(0) ? sqrt(s2) : T(0);
}

// coefficients.jl:264-288
template <class T>
__device__ __forceinline__ T cap_factor(T I, T Q, T V, T fmax_) {
    if (!(I > T(0))) return (Q == T(0) && V == T(0)) ? T(1) : T(0);
    T s = pow2_below(fmax(fabs(I), fmax(fabs(Q), fabs(V))));
    T Ih = I / s, q = Q / s, v = V / s;
    T qv = q * q + v * v;
    T p = qv > T(0) ? sqrt(qv) : T(0);
    return p > fmax_ * Ih ? fmax_ * Ih / p : T(1);
}

// ---- frames.jl ------------------------------------------------------------------------------------

// What a sample contributes to every splat's frame: the BL contravariant momentum p^mu, its ZAMO
// components, and the inverse tetrad (Krang's metric_uu, jac_zamo_u_bl_d, jac_bl_u_zamo_d).
template <class T>
struct SampleFrame {
    T pu[4], pz[4];
    T lapse_inv, om_lapse, sDS, misS, ivarpi;   // jac_bl_u_zamo_d entries
    T r, sth, cth, a;
};

template <class T>
__device__ __forceinline__ SampleFrame<T> sample_frame(T a, T r, T th, T sth, T cth, T eta, T lam, bool nur, bool nuth) {
    SampleFrame<T> F;
    T S = r * r + a * a * cth * cth, D = r * r - T(2) * r + a * a;
    T A = sq(r * r + a * a) - a * a * D * sth * sth;
    // momentum_bl_d (frames.jl:93-97) with safe square roots
    T Pr = r * r + a * a - a * lam;
    T R = Pr * Pr - D * (eta + (lam - a) * (lam - a));
    T Th = eta + a * a * cth * cth - lam * lam * cth * cth / (sth * sth);
    T pr = (nur ? T(1) : T(-1)) * (R > T(0) ? sqrt(R) : T(0)) / D;
    T pth = (nuth ? T(1) : T(-1)) * (Th > T(0) ? sqrt(Th) : T(0));
    T pd[4] = {T(-1), pr, pth, lam};
    // metric_uu
    T gtt = -A / (S * D), gtp = -T(2) * a * r / (S * D), grr = D / S, gthth = T(1) / S, gpp = (D - a * a * sth * sth) / (S * D * sth * sth);
    F.pu[0] = gtt * pd[0] + gtp * pd[3];
    F.pu[1] = grr * pd[1];
    F.pu[2] = gthth * pd[2];
    F.pu[3] = gtp * pd[0] + gpp * pd[3];
    // ZAMO tetrad (t, r, phi, -theta)
    T lapse = sqrt(S * D / A), om = T(2) * a * r / A, varpi = sqrt(A / S) * sth;
    F.pz[0] = lapse * F.pu[0];
    F.pz[1] = sqrt(S / D) * F.pu[1];
    F.pz[2] = -varpi * om * F.pu[0] + varpi * F.pu[3];
    F.pz[3] = -sqrt(S) * F.pu[2];
    F.lapse_inv = T(1) / lapse; F.om_lapse = om / lapse; F.sDS = sqrt(D / S); F.misS = -T(1) / sqrt(S); F.ivarpi = T(1) / varpi;
    F.r = r; F.sth = sth; F.cth = cth; F.a = a;
    return F;
}

// g, the pitch-angle cosine, the screen angle chi and the rotation by 2 chi (s2c = sin 2chi, c2c =
// cos 2chi). In FP32 the rotation comes straight from the Walker-Penrose components (x, y) of
// chi = atan2(y, x): cos 2chi = (x^2 - y^2) / (x^2 + y^2), sin 2chi = 2 x y / (x^2 + y^2), with
// no angle formed; in FP64 chi is formed as the reference forms it.
template <class T>
struct LFrame { T g, cosB, chi, s2c, c2c; };

// frames.jl:108-128 for one splat (fluid ZAMO 3-velocity u, unit field direction bh)
template <class T>
__device__ __forceinline__ LFrame<T> local_frame(const SampleFrame<T>& F, T u1, T u2, T u3, T bx, T by, T bz, bool bzero,
                                                 T alpha, T beta, T a_sin_tho) {
    T u2s = u1 * u1 + u2 * u2 + u3 * u3;
    T gam = sqrt(T(1) + u2s), q = T(1) / (gam + T(1));
    // p_f = Lambda(u) p_zamo
    T pf0 = gam * F.pz[0] - u1 * F.pz[1] - u2 * F.pz[2] - u3 * F.pz[3];
    T ud = u1 * F.pz[1] + u2 * F.pz[2] + u3 * F.pz[3];
    T pf1 = -u1 * F.pz[0] + F.pz[1] + u1 * ud * q;
    T pf2 = -u2 * F.pz[0] + F.pz[2] + u2 * ud * q;
    T pf3 = -u3 * F.pz[0] + F.pz[3] + u3 * ud * q;
    T g = T(1) / pf0;
    T k0 = pf1 * g, k1 = pf2 * g, k2 = pf3 * g;
    if (bzero) { bx = T(0); by = T(0); bz = T(1); }
    T cosB = k0 * bx + k1 * by + k2 * bz;
    T f0 = k1 * bz - k2 * by, f1 = k2 * bx - k0 * bz, f2 = k0 * by - k1 * bx;
    T fn = sqrt(f0 * f0 + f1 * f1 + f2 * f2);
    if (!(fn > T(0))) return {g, cosB, T(0), T(0), T(1)};
    f0 /= fn; f1 /= fn; f2 /= fn;
    // f_zamo = Lambda(-u) (0, f)
    T fd = u1 * f0 + u2 * f1 + u3 * f2;
    T fz0 = fd;
    T fz1 = f0 + u1 * fd * q, fz2 = f1 + u2 * fd * q, fz3 = f2 + u3 * fd * q;
    // f_bl = jac_bl_u_zamo_d f_zamo
    T ft = F.lapse_inv * fz0, fr = F.sDS * fz1, fth = F.misS * fz3, fph = F.om_lapse * fz0 + F.ivarpi * fz2;
    // walker_penrose (frames.jl:62-70)
    const T a = F.a, r = F.r, sth = F.sth, cth = F.cth;
    T Aw = F.pu[0] * fr - F.pu[1] * ft + a * sth * sth * (F.pu[1] * fph - F.pu[3] * fr);
    T Bw = ((r * r + a * a) * (F.pu[3] * fth - F.pu[2] * fph) - a * (F.pu[0] * fth - F.pu[2] * ft)) * sth;
    T kk1 = Aw * r - Bw * a * cth, kk2 = -(Aw * a * cth + Bw * r);
    // screen_direction (frames.jl:78-81)
    T mu = -(alpha + a_sin_tho);
    T ea = beta * kk2 - mu * kk1, eb = beta * kk1 + mu * kk2;
    if constexpr (is_f32<T>) {
        const T y = -ea, x = eb;
        const T r2 = x * x + y * y;
        if (!(r2 > T(0))) return {g, cosB, T(0), T(0), T(1)};
        const T ir = T(1) / r2;
        return {g, cosB, T(0), T(2) * x * y * ir, (x * x - y * y) * ir};
    } else {
        const T chi = atan2(-ea, eb);
        return {g, cosB, chi, sin(T(2) * chi), cos(T(2) * chi)};
    }
}

// ---- step.jl --------------------------------------------------------------------------------------

// M_n(a) = int_0^1 t^n e^{-at} dt for n = 0..9 (step.jl:239-268); the series coefficients
// (-1)^m / (m! (n + m + 1)) are generated on the host into constant memory.
struct MomentCoeffs { double c[10][24]; float cf[10][24]; };

template <class T>
__device__ __forceinline__ T mcoef(const MomentCoeffs& MC, int n, int m) {
    if constexpr (is_f32<T>) return T(MC.cf[n][m]);
    else return T(MC.c[n][m]);
}

template <class T>
__device__ __forceinline__ T moment_n(const MomentCoeffs& MC, T a, int n) {
    if (fabs(a) < T(1)) {
        T s = mcoef<T>(MC, n, 23);
#pragma unroll
        for (int m = 22; m >= 0; --m) s = fma(a, s, mcoef<T>(MC, n, m));
        return s;
    }
    T e = exp(-a);
    T M = (T(1) - e) / a;
    for (int q = 1; q <= n; ++q) M = (T(q) * M - e) / a;
    return M;
}
template <class T>
__device__ __forceinline__ void moments(const MomentCoeffs& MC, T a, T M[10]) {
    if (fabs(a) < T(1)) {
#pragma unroll
        for (int n = 0; n < 10; ++n) {
            T s = mcoef<T>(MC, n, 23);
#pragma unroll
            for (int m = 22; m >= 0; --m) s = fma(a, s, mcoef<T>(MC, n, m));
            M[n] = s;
        }
    } else {
        T e = exp(-a);
        M[0] = (T(1) - e) / a;
#pragma unroll
        for (int n = 1; n < 10; ++n) M[n] = (T(n) * M[n - 1] - e) / a;
    }
}
// FP32: one out-of-line copy; for |a| < 1 the series of M_9 and the downward recurrence
// M_{n-1} = (a M_n + e^{-a}) / n, stable for |a| < 1 (each step scales the error by |a| / n)
__device__ __noinline__ void moments_f32(const MomentCoeffs& MC, float a, float* M) {
    if (fabsf(a) < 1.f) {
        float s = MC.cf[9][23];
#pragma unroll
        for (int m = 22; m >= 0; --m) s = fmaf(a, s, MC.cf[9][m]);
        M[9] = s;
        const float e = __expf(-a);
#pragma unroll
        for (int n = 9; n >= 1; --n) M[n - 1] = (a * M[n] + e) * (1.f / float(n));
    } else {
        float e = __expf(-a);
        M[0] = (1.f - e) / a;
#pragma unroll
        for (int n = 1; n < 10; ++n) M[n] = (float(n) * M[n - 1] - e) / a;
    }
}
template <> __device__ __forceinline__ void moments<float>(const MomentCoeffs& MC, float a, float M[10]) { moments_f32(MC, a, M); }

template <class T> __device__ __forceinline__ T phi_fn(const MomentCoeffs& MC, T a) {
    if (fabs(a) < T(1)) return moment_n(MC, a, 0);
    if constexpr (is_f32<T>) return (T(1) - fexp(-a)) / a;   // |a| >= 1: no cancellation
    return -expm1(-a) / a;
}

// step.jl:147-153, in the scalar type of T (duals compare their values)
template <class T> __device__ __forceinline__ scalar_t<T> lin_thr() {
    if constexpr (is_f32<T>) return 1e-25f;
    else return 1e-200;
}
template <class T> __device__ __forceinline__ scalar_t<T> cub_thr() {
    if constexpr (is_f32<T>) return 1.1920929e-7f / 20.0f;
    else return 1e-17;
}

template <class T>
__device__ __forceinline__ T sinhc_excess(T b) {
    if (fabs(b) < T(0.1)) { T b2 = b * b; return b2 / T(6) * (T(1) + b2 / T(20) * (T(1) + b2 / T(42) * (T(1) + b2 / T(72) * (T(1) + b2 / T(110))))); }
    return sinh(b) / b - T(1);
}
template <class T>
__device__ __forceinline__ T sinc_deficit(T b) {
    if (fabs(b) < T(0.1)) { T b2 = b * b; return b2 / T(6) * (T(1) - b2 / T(20) * (T(1) - b2 / T(42) * (T(1) - b2 / T(72) * (T(1) - b2 / T(110))))); }
    return T(1) - sin(b) / b;
}

// K' = [0 aQ aU aV; aQ 0 rV -rU; aU -rV 0 rQ; aV rU -rQ 0] (row-major), its square and cube.
template <class T>
__device__ __forceinline__ void kmats(T aQ, T aU, T aV, T rQ, T rU, T rV, T K1[16], T K2[16], T K3[16]) {
    K1[0] = 0; K1[1] = aQ; K1[2] = aU; K1[3] = aV;
    K1[4] = aQ; K1[5] = 0; K1[6] = rV; K1[7] = -rU;
    K1[8] = aU; K1[9] = -rV; K1[10] = 0; K1[11] = rQ;
    K1[12] = aV; K1[13] = rU; K1[14] = -rQ; K1[15] = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            T s = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k) s += K1[4 * i + k] * K1[4 * k + j];
            K2[4 * i + j] = s;
        }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            T s = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k) s += K2[4 * i + k] * K1[4 * k + j];
            K3[4 * i + j] = s;
        }
}

// The step operator (step.jl:45-124): O = exp(-K D) and Ej = int_0^D exp(-K u) du, both 4x4 row-major.
template <class T>
__device__ __forceinline__ void step_operator(const MomentCoeffs& MC, const T al[4], const T rh[3], T Dlen, T O[16], T Ej[16]) {
    const T s = pow2_below(Dlen);
    const T D = Dlen / s;
    T aI = al[0] * s, aQ = al[1] * s, aU = al[2] * s, aV = al[3] * s;
    T rQ = rh[0] * s, rU = rh[1] * s, rV = rh[2] * s;
    T a2 = aQ * aQ + aU * aU + aV * aV;
    T r2 = rQ * rQ + rU * rU + rV * rV;
    T a = aI * D;
    T K1[16], K2[16], K3[16];
    if ((a2 + r2) * D * D < lin_thr<T>()) {
        T e = exp(-a);
        T ph = phi_fn(MC, a), m1 = moment_n(MC, a, 1);
        K1[0] = 0; K1[1] = aQ; K1[2] = aU; K1[3] = aV; K1[4] = aQ; K1[5] = 0; K1[6] = rV; K1[7] = -rU;
        K1[8] = aU; K1[9] = -rV; K1[10] = 0; K1[11] = rQ; K1[12] = aV; K1[13] = rU; K1[14] = -rQ; K1[15] = 0;
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            T id = (i % 5 == 0) ? T(1) : T(0);
            O[i] = e * (id - D * K1[i]);
            Ej[i] = D * (ph * id - (D * m1) * K1[i]);
        }
    } else {
        kmats(aQ, aU, aV, rQ, rU, rV, K1, K2, K3);
        T ar = aQ * rQ + aU * rU + aV * rV;
        T h = (a2 - r2) / T(2);
        T rt2 = h * h + ar * ar;
        T root = rt2 > T(0) ? sqrt(rt2) : T(0);
        T L1sq, L2sq;
        if (h >= T(0)) { L1sq = h + root; L2sq = L1sq > T(0) ? ar * ar / L1sq : T(0); }
        else { L2sq = root - h; L1sq = L2sq > T(0) ? ar * ar / L2sq : T(0); }
        T L1 = L1sq > T(0) ? sqrt(L1sq) : T(0), L2 = L2sq > T(0) ? sqrt(L2sq) : T(0);
        T b1 = L1 * D, b2 = L2 * D;
        T Th = L1sq + L2sq;
        if (Th * D * D * (T(1) + (a2 + r2) * D * D) < cub_thr<T>()) {
            T e = exp(-a);
            T M[10];
            moments(MC, a, M);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                T id = (i % 5 == 0) ? T(1) : T(0);
                O[i] = e * (id - D * K1[i] + (D * D / T(2)) * K2[i] - (D * D * D / T(6)) * K3[i]);
                Ej[i] = D * (M[0] * id - (D * M[1]) * K1[i] + (D * D * M[2] / T(2)) * K2[i] - (D * D * D * M[3] / T(6)) * K3[i]);
            }
        } else {
            T e = exp(-a);
            T ecosh, esinhb, ecoshm1;
            if (b1 < T(1)) {
                T sh = sinh(b1 / T(2));
                ecosh = e * cosh(b1);
                esinhb = e * (fabs(b1) < T(0.1) ? T(1) + sinhc_excess(b1) : sinh(b1) / b1);
                ecoshm1 = e * T(2) * sh * sh;
            } else {
                T em = exp(-(a - b1)), ep = exp(-(a + b1));
                ecosh = (em + ep) / T(2); esinhb = (em - ep) / (T(2) * b1); ecoshm1 = (em - T(2) * e + ep) / T(2);
            }
            T sb2 = sin(b2), cb2 = cos(b2), sh2 = sin(b2 / T(2));
            T c0 = (L2sq * ecosh + L1sq * e * cb2) / Th;
            T c2 = (ecoshm1 + e * T(2) * sh2 * sh2) / Th;
            T sincb2 = fabs(b2) < T(0.1) ? T(1) - sinc_deficit(b2) : sb2 / b2;
            T so = D * esinhb, sn = D * e * sincb2;
            // the integrals (step.jl:116-121)
            T M[10];
            moments(MC, a, M);
            T ph_a = fabs(a) < T(1) ? M[0] : -expm1(-a) / a;
            T icoshm1 = b1 < T(0.1) ? b1 * b1 * (M[2] / T(2) + b1 * b1 * (M[4] / T(24) + b1 * b1 * (M[6] / T(720) + b1 * b1 * M[8] / T(40320))))
                                   : (phi_fn(MC, a - b1) + phi_fn(MC, a + b1)) / T(2) - ph_a;
            T vser = b2 * b2 * (M[2] / T(2) - b2 * b2 * (M[4] / T(24) - b2 * b2 * (M[6] / T(720) - b2 * b2 * M[8] / T(40320))));
            T icos_closed = (a - e * (a * cb2 - b2 * sb2)) / (a * a + b2 * b2);
            T iversin = b2 < T(0.1) ? vser : ph_a - icos_closed;
            T icos = b2 < T(0.1) ? ph_a - vser : icos_closed;
            T sdser = b2 * b2 * (M[3] / T(6) - b2 * b2 * (M[5] / T(120) - b2 * b2 * (M[7] / T(5040) - b2 * b2 * M[9] / T(362880))));
            T isinc = b2 < T(0.1) ? M[1] - sdser : (T(1) - e * (a * sb2 / b2 + cb2)) / (a * a + b2 * b2);
            T ishx = b1 < T(0.1) ? b1 * b1 * (M[3] / T(6) + b1 * b1 * (M[5] / T(120) + b1 * b1 * (M[7] / T(5040) + b1 * b1 * M[9] / T(362880))))
                                : (phi_fn(MC, a - b1) - phi_fn(MC, a + b1)) / (T(2) * b1) - M[1];
            T Ich = D * (ph_a + icoshm1);
            T Ic = D * icos;
            T Ish = D * D * (M[1] + ishx);
            T Is = D * D * isinc;
            T C0 = (L2sq * Ich + L1sq * Ic) / Th;
            T C2 = D * (icoshm1 + iversin) / Th;
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                T id = (i % 5 == 0) ? T(1) : T(0);
                T M2 = (L1sq * K1[i] - K3[i]) / Th;
                T M3 = (L2sq * K1[i] + K3[i]) / Th;
                O[i] = c0 * id + c2 * K2[i] - so * M3 - sn * M2;
                Ej[i] = C0 * id + C2 * K2[i] - Ish * M3 - Is * M2;
            }
        }
    }
    // the rescaled emission integral (s is a power of two: exact)
#pragma unroll
    for (int i = 0; i < 16; ++i) Ej[i] = s * Ej[i];
}

// The exact step (step.jl:27-30): O = exp(-K D) and E = (int_0^D exp(-K u) du) j.
template <class T>
__device__ __forceinline__ void transfer_step(const MomentCoeffs& MC, const T j4[4], const T al[4], const T rh[3], T Dlen,
                                              T O[16], T E[4]) {
    T Ej[16];
    step_operator(MC, al, rh, Dlen, O, Ej);
#pragma unroll
    for (int i = 0; i < 4; ++i) E[i] = Ej[4 * i] * j4[0] + Ej[4 * i + 1] * j4[1] + Ej[4 * i + 2] * j4[2] + Ej[4 * i + 3] * j4[3];
}

// the coefficients (o_n, e_n) of the rescaled step at the scaled invariants; same branches and
// thresholds as step_operator
template <class TD>
__device__ __forceinline__ void step_coefficients(const MomentCoeffs& MC, TD a, TD a2, TD r2, TD ar, scalar_t<TD> D, TD o[4], TD e[4]) {
    using S = scalar_t<TD>;
    if ((a2 + r2) * D * D < lin_thr<TD>()) {
        const TD ex = exp(-a), ph = phi_fn(MC, a), m1 = moment_n(MC, a, 1);
        o[0] = ex; o[1] = -D * ex; o[2] = TD(S(0)); o[3] = TD(S(0));
        e[0] = D * ph; e[1] = -(D * D) * m1; e[2] = TD(S(0)); e[3] = TD(S(0));
        return;
    }
    const TD h = (a2 - r2) / S(2);
    const TD rt2 = h * h + ar * ar;
    const TD root = rt2 > S(0) ? sqrt(rt2) : TD(S(0));
    TD L1sq, L2sq;
    if (h >= S(0)) { L1sq = h + root; L2sq = L1sq > S(0) ? ar * ar / L1sq : TD(S(0)); }
    else { L2sq = root - h; L1sq = L2sq > S(0) ? ar * ar / L2sq : TD(S(0)); }
    const TD L1 = L1sq > S(0) ? sqrt(L1sq) : TD(S(0)), L2 = L2sq > S(0) ? sqrt(L2sq) : TD(S(0));
    const TD b1 = L1 * D, b2 = L2 * D;
    const TD Th = L1sq + L2sq;
    const TD ex = fexp(-a);
    TD M[10];
    moments(MC, a, M);
    if (Th * D * D * ((a2 + r2) * D * D + S(1)) < cub_thr<TD>()) {
        o[0] = ex; o[1] = -D * ex; o[2] = (D * D / S(2)) * ex; o[3] = -(D * D * D / S(6)) * ex;
        e[0] = D * M[0]; e[1] = -(D * D) * M[1]; e[2] = (D * D * D / S(2)) * M[2]; e[3] = -(D * D * D * D / S(6)) * M[3];
        return;
    }
    TD ecosh, esinhb, ecoshm1;
    if (b1 < S(1)) {
        const TD sh = sinh(b1 / S(2));
        ecosh = ex * cosh(b1);
        esinhb = ex * (fabs(b1) < S(0.1) ? sinhc_excess(b1) + S(1) : sinh(b1) / b1);
        ecoshm1 = ex * S(2) * sh * sh;
    } else {
        const TD em = fexp(-(a - b1)), ep = fexp(-(a + b1));
        ecosh = (em + ep) / S(2); esinhb = (em - ep) / (S(2) * b1); ecoshm1 = (em - S(2) * ex + ep) / S(2);
    }
    TD sb2, cb2, sh2;
    if constexpr (is_f32<TD>) {
        // one reduced hardware sine/cosine of the half angle: sin b2 = 2 s c, cos b2 = 1 - 2 s^2
        TD ch2;
        fsincos(b2 / S(2), sh2, ch2);
        sb2 = S(2) * sh2 * ch2;
        cb2 = S(1) - S(2) * sh2 * sh2;
    } else {
        sb2 = sin(b2); cb2 = cos(b2); sh2 = sin(b2 / S(2));
    }
    const TD c0 = (L2sq * ecosh + L1sq * ex * cb2) / Th;
    const TD c2 = (ecoshm1 + ex * S(2) * sh2 * sh2) / Th;
    const TD sincb2 = fabs(b2) < S(0.1) ? S(1) - sinc_deficit(b2) : sb2 / b2;
    const TD so = D * esinhb, sn = D * ex * sincb2;
    const TD ph_a = fabs(a) < S(1) ? M[0] : (S(1) - ex) / a;   // |a| >= 1: no cancellation
    const TD icoshm1 = b1 < S(0.1) ? b1 * b1 * (M[2] / S(2) + b1 * b1 * (M[4] / S(24) + b1 * b1 * (M[6] / S(720) + b1 * b1 * M[8] / S(40320))))
                                   : (phi_fn(MC, a - b1) + phi_fn(MC, a + b1)) / S(2) - ph_a;
    const TD vser = b2 * b2 * (M[2] / S(2) - b2 * b2 * (M[4] / S(24) - b2 * b2 * (M[6] / S(720) - b2 * b2 * M[8] / S(40320))));
    const TD icos_closed = (a - ex * (a * cb2 - b2 * sb2)) / (a * a + b2 * b2);
    const TD iversin = b2 < S(0.1) ? vser : ph_a - icos_closed;
    const TD icos = b2 < S(0.1) ? ph_a - vser : icos_closed;
    const TD sdser = b2 * b2 * (M[3] / S(6) - b2 * b2 * (M[5] / S(120) - b2 * b2 * (M[7] / S(5040) - b2 * b2 * M[9] / S(362880))));
    const TD isinc = b2 < S(0.1) ? M[1] - sdser : (S(1) - ex * (a * sb2 / b2 + cb2)) / (a * a + b2 * b2);
    const TD ishx = b1 < S(0.1) ? b1 * b1 * (M[3] / S(6) + b1 * b1 * (M[5] / S(120) + b1 * b1 * (M[7] / S(5040) + b1 * b1 * M[9] / S(362880))))
                                : (phi_fn(MC, a - b1) - phi_fn(MC, a + b1)) / (S(2) * b1) - M[1];
    const TD Ich = D * (ph_a + icoshm1);
    const TD Ic = D * icos;
    const TD Ish = D * D * (M[1] + ishx);
    const TD Is = D * D * isinc;
    const TD C0 = (L2sq * Ich + L1sq * Ic) / Th;
    const TD C2 = D * (icoshm1 + iversin) / Th;
    o[0] = c0; o[1] = -(so * L2sq + sn * L1sq) / Th; o[2] = c2; o[3] = (sn - so) / Th;
    e[0] = C0; e[1] = -(Ish * L2sq + Is * L1sq) / Th; e[2] = C2; e[3] = (Is - Ish) / Th;
}

// <x, G_theta y> for the six sparse generators G = dK/dtheta, theta = aQ, aU, aV, rQ, rU, rV
template <class T>
__device__ __forceinline__ void kgen_forms(const T x[4], const T y[4], T out[6]) {
    out[0] = x[0] * y[1] + x[1] * y[0];
    out[1] = x[0] * y[2] + x[2] * y[0];
    out[2] = x[0] * y[3] + x[3] * y[0];
    out[3] = x[2] * y[3] - x[3] * y[2];
    out[4] = x[3] * y[1] - x[1] * y[3];
    out[5] = x[1] * y[2] - x[2] * y[1];
}

template <class T>
__device__ __forceinline__ void kmul(const T K[16], const T v[4], T out[4]) {
#pragma unroll
    for (int i = 0; i < 4; ++i) out[i] = K[4 * i] * v[0] + K[4 * i + 1] * v[1] + K[4 * i + 2] * v[2] + K[4 * i + 3] * v[3];
}
template <class T>
__device__ __forceinline__ void kmul_t(const T K[16], const T v[4], T out[4]) {
#pragma unroll
    for (int i = 0; i < 4; ++i) out[i] = K[i] * v[0] + K[4 + i] * v[1] + K[8 + i] * v[2] + K[12 + i] * v[3];
}
template <class T>
__device__ __forceinline__ T dot4(const T x[4], const T y[4]) { return x[0] * y[0] + x[1] * y[1] + x[2] * y[2] + x[3] * y[3]; }

// The exact step in its structured form: O = sum_n o_n K^n, E = s sum_n e_n K^n j with the
// coefficients of step_coefficients, K the rescaled matrix and s the power-of-two rescaling: the same
// operator as transfer_step (the same branches and thresholds), with one assembly for all branches.
template <class T>
__device__ __forceinline__ void transfer_step_structured(const MomentCoeffs& MC, const T j4[4], const T al[4], const T rh[3], T Dl, T O[16],
                                                         T E[4]) {
    const T s = pow2_below(Dl);
    const T D = Dl / s;
    const T aI = al[0] * s, aQ = al[1] * s, aU = al[2] * s, aV = al[3] * s, rQ = rh[0] * s, rU = rh[1] * s, rV = rh[2] * s;
    T o[4], e[4];
    step_coefficients(MC, aI * D, aQ * aQ + aU * aU + aV * aV, rQ * rQ + rU * rU + rV * rV, aQ * rQ + aU * rU + aV * rV, D, o, e);
    T K[16];
    K[0] = 0; K[1] = aQ; K[2] = aU; K[3] = aV; K[4] = aQ; K[5] = 0; K[6] = rV; K[7] = -rU;
    K[8] = aU; K[9] = -rV; K[10] = 0; K[11] = rQ; K[12] = aV; K[13] = rU; K[14] = -rQ; K[15] = 0;
    T K2[16];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) K2[4 * i + jj] = K[4 * i] * K[jj] + K[4 * i + 1] * K[4 + jj] + K[4 * i + 2] * K[8 + jj] + K[4 * i + 3] * K[12 + jj];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
            const T k3 = K2[4 * i] * K[jj] + K2[4 * i + 1] * K[4 + jj] + K2[4 * i + 2] * K[8 + jj] + K2[4 * i + 3] * K[12 + jj];
            O[4 * i + jj] = ((i == jj) ? o[0] : T(0)) + o[1] * K[4 * i + jj] + o[2] * K2[4 * i + jj] + o[3] * k3;
        }
    T Kj[4], K2j[4], K3j[4];
    kmul(K, j4, Kj); kmul(K, Kj, K2j); kmul(K, K2j, K3j);
#pragma unroll
    for (int i = 0; i < 4; ++i) E[i] = s * (e[0] * j4[i] + e[1] * Kj[i] + e[2] * K2j[i] + e[3] * K3j[i]);
}

// ---- splats -------------------------------------------------------------------------------------

// Gaussian x temporal-envelope exponent and weight of splat row `p` (FP64 table cast to T) at
// time t and position x (Splats.jl:58-93, polarized.jl:22-29, 110-120). Returns false when the
// support-sphere cull rejects the point (no weight evaluated), in which case q is untouched.
template <class T>
__device__ __forceinline__ bool splat_exponent(const T* p, T t, T x, T y, T z, bool cull, T& q) {
    T ph = p[ST_OMEGA] * (t - p[ST_T0]);
    T sp, cp;
    fsincos(ph, sp, cp);
    T cx = p[ST_CX] * cp - p[ST_CY] * sp, cy = p[ST_CX] * sp + p[ST_CY] * cp;
    T d0 = x - cx, d1 = y - cy, d2 = z - p[ST_CZ];
    if (cull && d0 * d0 + d1 * d1 + d2 * d2 > p[ST_SUPP]) return false;
    T dr0 = d0 * cp + d1 * sp, dr1 = -d0 * sp + d1 * cp, dr2 = d2;
    T u0 = p[ST_R0] * dr0 + p[ST_R3] * dr1 + p[ST_R6] * dr2;
    T u1 = p[ST_R1] * dr0 + p[ST_R4] * dr1 + p[ST_R7] * dr2;
    T u2 = p[ST_R2] * dr0 + p[ST_R5] * dr1 + p[ST_R8] * dr2;
    T e0 = u0 * p[ST_ES1], e1 = u1 * p[ST_ES2], e2 = u2 * p[ST_ES3];
    T tt = (t - p[ST_T0]) * p[ST_INVW];
    q = (e0 * e0 + e1 * e1 + e2 * e2 + tt * tt) / T(2);
    return true;
}

// knot_centre (trajectories.jl:93-111): the centre interpolated linearly between the knots at time t,
// clamped to the end knots; kn = [times (nk), x (nk), y (nk), z (nk)] with increasing times
template <class T>
__device__ __forceinline__ void knot_centre(const T* kn, int nk, T t, T& cx, T& cy, T& cz) {
    const T* ts = kn;
    const T *X = kn + nk, *Y = kn + 2 * nk, *Z = kn + 3 * nk;
    if (t <= ts[0]) { cx = X[0]; cy = Y[0]; cz = Z[0]; return; }
    if (t >= ts[nk - 1]) { cx = X[nk - 1]; cy = Y[nk - 1]; cz = Z[nk - 1]; return; }
    int k = 0;
    while (k < nk - 2 && ts[k + 1] <= t) ++k;
    const T w = (t - ts[k]) / (ts[k + 1] - ts[k]);
    cx = (T(1) - w) * X[k] + w * X[k + 1];
    cy = (T(1) - w) * Y[k] + w * Y[k + 1];
    cz = (T(1) - w) * Z[k] + w * Z[k + 1];
}

// The weight exponent of a knot splat (KnotSplats element, trajectories.jl:113-129): the centre from
// its knots at the emission time, no pattern rotation and no support cull; knots = the knot array.
template <class T>
__device__ __forceinline__ void knot_exponent(const T* p, const T* knots, T t, T x, T y, T z, T& q) {
    T cx, cy, cz;
    knot_centre(knots + int(value_of(p[ST_KOFF])), int(value_of(p[ST_NK])), t, cx, cy, cz);
    const T d0 = x - cx, d1 = y - cy, d2 = z - cz;
    const T u0 = p[ST_R0] * d0 + p[ST_R3] * d1 + p[ST_R6] * d2;
    const T u1 = p[ST_R1] * d0 + p[ST_R4] * d1 + p[ST_R7] * d2;
    const T u2 = p[ST_R2] * d0 + p[ST_R5] * d1 + p[ST_R8] * d2;
    const T e0 = u0 * p[ST_ES1], e1 = u1 * p[ST_ES2], e2 = u2 * p[ST_ES3];
    const T tt = (t - p[ST_T0]) * p[ST_INVW];
    q = (e0 * e0 + e1 * e1 + e2 * e2 + tt * tt) / T(2);
}

// The exponent of any splat of a polarized scene: false when the support sphere culls it.
template <class T>
__device__ __forceinline__ bool any_exponent(const T* p, const T* knots, T t, T x, T y, T z, T& q) {
    if (int(value_of(p[ST_KIND])) == KS_KNOT21) {
        const T dx = x - p[ST_CX], dy = y - p[ST_CY], dz = z - p[ST_CZ];
        if (dx * dx + dy * dy + dz * dz > p[ST_RHO]) return false;   // outside the knots' bounding sphere
        knot_exponent(p, knots, t, x, y, z, q);
        return true;
    }
    return splat_exponent(p, t, x, y, z, true, q);
}

}  // namespace ks
