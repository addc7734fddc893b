// ks_plan.cuh -- the FP64 per-ray plan: root cases (K0), per-ray constants (K1) and the anchor table.
//
// The reference builds Krang's SlowLightIntensityPixel per pixel (pixel_constants.jl:110-157) and
// then, at the top of every per-ray kernel launch, the recurrence and quadrature constants
// (quadrature.jl:232-243) and one closed-form anchor every M samples (quadrature.jl:248, 283-291).
// Here everything that depends only on (a, theta_o, camera, N, M) is built once per regenerate in
// FP64 and stored structure-of-arrays in sorted-slot order, so that the march kernels read it
// coalesced and never evaluate an elliptic function:
//   * plan fields (PF_*): one FP64 array of stride `npad` per field;
//   * anchors: one 96-byte record per anchor (k = 1 + m * M_anchor), ray-major with CSR offsets:
//     the Jacobi states of r and theta, t~ and phi, and the validity flag.
// The anchors' t~ and phi are the Mino-time integrals of the rates split as in quadrature.jl:1-35
// (large-r, horizon and polar-axis parts in closed form) with the smooth remainder integrated by
// 16-point Gauss-Legendre panels, t~ regularized by dropping r_obs + 2 ln r_obs and phi(0) = 0.
#pragma once
#include "ks_elliptic.cuh"

namespace ks {

template <class T>
struct SpacetimeT {
    T a, thetao, rp, rmn, rh, abscos, cos2;
    int N, M;        // N: samples per ray (with uneven counts, the largest)
    // uneven counts: N_j = clamp(64 ceil(density tau_total_j / 64), nmin, N); density 0 = uniform N
    double density;
    int nmin;
};
using Spacetime = SpacetimeT<double>;

enum PlanField {
    PF_ALPHA, PF_BETA, PF_ETA, PF_LAM, PF_NUMREALS, PF_CASE,
    PF_K, PF_C, PF_FO, PF_MAP0, PF_MAP1, PF_MAP2, PF_MAP3,
    PF_TAU_VALID, PF_TAU_TOTAL, PF_DTAU,
    PF_PMU, PF_PSCALE, PF_TEMPFAC, PF_POFFSET, PF_SQRTUP, PF_UM, PF_UPMUM, PF_PSIGN, PF_VORTICAL, PF_GTHO,
    PF_SP, PF_SM, PF_QT, PF_QTM, PF_QPHI, PF_QPHIM, PF_R4, PF_SCATTER,
    PF_QC, PF_QN, PF_SQRTEPS, PF_GC, PF_MP, PF_K2,
    PF_VABSALPHA, PF_VALPHA2, PF_VABSBETA,
    PF_DR_SN, PF_DR_CN, PF_DR_DN, PF_DTH_SN, PF_DTH_CN, PF_DTH_DN,
    PF_TURN_K,                                   // sample k whose interval (k-1, k) holds fo (scattering), else -1
    PF_P1R_SN, PF_P1R_CN, PF_P1R_DN, PF_P1T_SN, PF_P1T_CN, PF_P1T_DN,   // direct states at (ta + fo)/2
    PF_P2R_SN, PF_P2R_CN, PF_P2R_DN, PF_P2T_SN, PF_P2T_CN, PF_P2T_DN,   // ... at (fo + tb)/2
    PF_PTT_SN, PF_PTT_CN, PF_PTT_DN,                                     // polar state at fo
    PF_MANCHOR, PF_NANCH,
    PF_R1RE, PF_R1IM, PF_R2RE, PF_R2IM, PF_R3RE, PF_R3IM, PF_R4RE, PF_R4IM,
    PF_NSAMP,                                    // samples of this ray
    PF_COUNT
};

// One anchor record (12 doubles = 96 bytes).
enum AnchorField { AF_XR_SN, AF_XR_CN, AF_XR_DN, AF_XT_SN, AF_XT_CN, AF_XT_DN, AF_T, AF_PHI, AF_OK,
                   AF_SEG_T, AF_SEG_PHI, AF_PAD, AF_COUNT };

template <class T> struct CplxT { T re, im; };

template <class T> KS_HD CplxT<T> cx(T r, T i) { return {r, i}; }
template <class T> KS_HD CplxT<T> cadd(CplxT<T> a, CplxT<T> b) { return {a.re + b.re, a.im + b.im}; }
template <class T> KS_HD CplxT<T> cmul(CplxT<T> a, CplxT<T> b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
template <class T> KS_HD CplxT<T> cdiv(CplxT<T> a, CplxT<T> b) {
    T d = b.re * b.re + b.im * b.im;
    return {(a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d};
}
template <class T> KS_HD T cabs_(CplxT<T> a) { return hypot(a.re, a.im); }
// principal square root of a real number as a complex number
template <class T> KS_HD CplxT<T> csqrt_real(T x) { return val(x) >= 0 ? CplxT<T>{sqrt(x), T(0.0)} : CplxT<T>{T(0.0), sqrt(-x)}; }
// principal cube root of a complex number
template <class T> KS_HD CplxT<T> ccbrt(CplxT<T> z) {
    T r = cabs_(z);
    if (val(r) == 0.0) return {T(0.0), T(0.0)};
    T th = atan2(z.im, z.re) / 3.0;
    T m = cbrt(r);
    return {m * cos(th), m * sin(th)};
}

// All the constants of one ray (sorted slot), built from the screen point; T = double for the
// geodesics, a dual number for their derivatives in (a, theta_o).
template <class T>
struct RayCT {
    T alpha, beta, eta, lam;
    T rre[4], rim[4];
    int numreals, rcase;
    T k, c, fo, map[4], tau_valid, tau_total;
    T pmu, pscale, tempfac, poffset, sqrt_up, um, up_m_um, psign; bool vortical; T gtho;
    T sp, sm, Qt, Qtm, Qphi, Qphim, r4, qC, qn, sqrt_eps, gc, mp, K2; bool scattering;
    T vabsalpha, valpha2, vabsbeta;
};
using RayC = RayCT<double>;

KS_HD double sgn(double x) { return x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0); }

// Mino time at which the inbound radial closed form reaches radius r (inverse of the r(X) maps,
// recurrence.jl:169-177): tau = fo - X / c.
template <class T>
KS_HD T mino_time_at(const RayCT<T>& R, T r) {
    T X;
    if (R.rcase == 2) {
        T r1 = R.rre[0], r3 = R.rre[2], r4 = R.rre[3];
        T s2 = (r3 - r1) * (r4 - r) / ((r4 - r1) * (r3 - r));
        X = ellip_f(asin(sqrt(fmax(T(0.0), fmin(T(1.0), s2)))), R.k);
    } else if (R.rcase == 3) {
        T cn = (R.map[0] - r * R.map[2]) / (r * R.map[3] - R.map[1]);
        X = ellip_f(acos(fmax(T(-1.0), fmin(T(1.0), cn))), R.k);
    } else {
        T w = -(r + R.map[1]) / R.map[0];
        T sc = (R.map[2] - w) / (1.0 + w * R.map[2]);
        T ph = atan(sc);
        if (val(ph) < 0.0) ph += kPi;
        X = ellip_f(ph, R.k);
    }
    return R.fo - X / R.c;
}

// Roots of the radial potential by the resolvent cubic (Gralla & Lupsasca 2020), the radial and
// polar closed-form constants (test/highprec_reference.jl:65-122, recurrence.jl:64-109, 207-237),
// the quadrature constants (quadrature.jl:68-97) and the visibility constants (recurrence.jl:293-298).
template <class T>
KS_HD RayCT<T> build_ray(const SpacetimeT<T>& st, T alpha, T beta) {
    RayCT<T> R;
    const T a = st.a, th = st.thetao;
    T ct = cos(th);
    R.alpha = alpha; R.beta = beta;
    R.eta = (alpha * alpha - a * a) * ct * ct + beta * beta;
    R.lam = -alpha * sin(th);
    const T eta = R.eta, lam = R.lam;
    // radial roots
    T A = a * a - eta - lam * lam;
    T B = 2.0 * (eta + (lam - a) * (lam - a));
    T Cc = -a * a * eta;
    T P = -A * A / 12.0 - Cc;
    T Q = -A / 3.0 * ((A / 6.0) * (A / 6.0) - Cc) - B * B / 8.0;
    T disc = (P / 3.0) * (P / 3.0) * (P / 3.0) + (Q / 2.0) * (Q / 2.0);
    CplxT<T> sq = csqrt_real(disc);
    CplxT<T> wp = ccbrt(cadd(cx(-Q / 2.0, T(0.0)), sq));
    CplxT<T> wm = val(cabs_(wp)) > 0.0 ? cdiv(cx(-P / 3.0, T(0.0)), wp) : ccbrt(cadd(cx(-Q / 2.0, T(0.0)), cx(-sq.re, -sq.im)));
    T xi0 = (wp.re + wm.re) - A / 3.0;
    T z = sqrt(fmax(xi0 / 2.0, T(0.0)));
    T arg12 = -A / 2.0 - z * z + B / (4.0 * z);
    T arg34 = -A / 2.0 - z * z - B / (4.0 * z);
    if (val(arg12) >= 0.0) { T s = sqrt(arg12); R.rre[0] = -z - s; R.rim[0] = T(0.0); R.rre[1] = -z + s; R.rim[1] = T(0.0); }
    else { T s = sqrt(-arg12); R.rre[0] = -z; R.rim[0] = -s; R.rre[1] = -z; R.rim[1] = s; }
    if (val(arg34) >= 0.0) { T s = sqrt(arg34); R.rre[2] = z - s; R.rim[2] = T(0.0); R.rre[3] = z + s; R.rim[3] = T(0.0); }
    else { T s = sqrt(-arg34); R.rre[2] = z; R.rim[2] = -s; R.rre[3] = z; R.rim[3] = s; }
    R.numreals = (val(arg12) >= 0.0 ? 2 : 0) + (val(arg34) >= 0.0 ? 2 : 0);
    R.rcase = R.numreals == 4 ? 2 : (R.numreals == 2 ? 3 : 4);
    const T inf = T(double(INFINITY));
    if (R.rcase == 2) {
        T r1 = R.rre[0], r2 = R.rre[1], r3 = R.rre[2], r4 = R.rre[3];
        T r31 = r3 - r1, r32 = r3 - r2, r41 = r4 - r1, r42 = r4 - r2;
        R.k = r32 * r41 / (r31 * r42);
        R.c = sqrt(r31 * r42) / 2.0;
        R.fo = 2.0 / sqrt(r31 * r42) * ellip_f(asin(sqrt(r31 / r41)), R.k);
        R.map[0] = r1; R.map[1] = r3; R.map[2] = r41; R.map[3] = r4 - r3;
        R.tau_total = 2.0 * R.fo;
        R.tau_valid = val(r4) < val(st.rh) ? mino_time_at(R, st.rh) : inf;
    } else if (R.rcase == 3) {
        T r1 = R.rre[0], r2 = R.rre[1];
        T r21 = r2 - r1;
        T dr32 = R.rre[2] - R.rre[1], di32 = R.rim[2] - R.rim[1];
        T dr31 = R.rre[2] - R.rre[0], di31 = R.rim[2] - R.rim[0];
        T Aa = sqrt(dr32 * dr32 + di32 * di32);
        T Bb = sqrt(dr31 * dr31 + di31 * di31);
        R.k = ((Aa + Bb) * (Aa + Bb) - r21 * r21) / (4.0 * Aa * Bb);
        R.c = sqrt(Aa * Bb);
        R.fo = ellip_f(acos((Aa - Bb) / (Aa + Bb)), R.k) / sqrt(Aa * Bb);
        R.map[0] = -Aa * r1 + Bb * r2; R.map[1] = Aa * r1 + Bb * r2; R.map[2] = Bb - Aa; R.map[3] = Aa + Bb;
        R.tau_valid = inf;
        R.tau_total = mino_time_at(R, st.rh);
    } else {
        T a1 = fabs(R.rim[3]), a2 = fabs(R.rim[1]);
        T b1 = R.rre[3], b2 = R.rre[1];
        T C = sqrt((a1 - a2) * (a1 - a2) + (b1 - b2) * (b1 - b2));
        T D = sqrt((a1 + a2) * (a1 + a2) + (b1 - b2) * (b1 - b2));
        R.k = 4.0 * C * D / ((C + D) * (C + D));
        R.c = (C + D) / 2.0;
        T g0 = sqrt(fmax((4.0 * a2 * a2 - (C - D) * (C - D)) / ((C + D) * (C + D) - 4.0 * a2 * a2), T(0.0)));
        R.fo = 2.0 / (C + D) * ellip_f(kPi / 2.0 + atan(g0), R.k);
        R.map[0] = a2; R.map[1] = b1; R.map[2] = g0; R.map[3] = T(0.0);
        R.tau_valid = inf;
        R.tau_total = mino_time_at(R, st.rh);
    }
    // polar constants, Krang's rounding (recurrence.jl:218-236)
    T Dth = (1.0 - (eta + lam * lam) / (a * a)) / 2.0;
    T dsc = sqrt(Dth * Dth + eta / (a * a));
    T up = Dth + dsc, um = Dth - dsc;
    T m = up / um;
    R.tempfac = 1.0 / sqrt(fabs(um * a * a));
    R.vortical = val(eta) < 0.0;
    double sb = sgn(val(beta));
    T kq;
    if (R.vortical) {
        kq = 1.0 - m;
        T arg = fmax(T(0.0), fmin(T(1.0), (ct * ct - um) / (up - um)));
        R.gtho = R.tempfac * ellip_f(asin(sqrt(arg)), kq);
        double sigma = val(th) > kPi / 2.0 ? -1.0 : 1.0;
        R.poffset = sigma * sb * R.gtho;
        R.psign = T(sigma);
    } else {
        kq = m;
        T arg = fmax(T(-1.0), fmin(T(1.0), ct / sqrt(up)));
        R.gtho = R.tempfac * ellip_f(asin(arg), kq);
        R.poffset = sb * R.gtho;
        R.psign = T(sb);
    }
    R.pmu = -kq / (1.0 - kq);
    R.pscale = sqrt(1.0 - kq);
    R.sqrt_up = sqrt(up); R.um = um; R.up_m_um = up - um;
    // quadrature constants
    T E = st.rp * st.rp + a * a - a * lam;
    T Em = st.rmn * st.rmn + a * a - a * lam;
    R.sp = -fabs(E); R.sm = -fabs(Em);
    R.Qt = (st.rp * st.rp + a * a) * E / (st.rp - st.rmn);
    R.Qtm = -(st.rmn * st.rmn + a * a) * Em / (st.rp - st.rmn);
    R.Qphi = a * (2.0 * st.rp - a * lam) / (st.rp - st.rmn);
    R.Qphim = -a * (2.0 * st.rmn - a * lam) / (st.rp - st.rmn);
    R.scattering = (R.rcase == 2) && !(val(R.tau_valid) < val(inf));
    R.r4 = R.rcase == 2 ? R.rre[3] : T(double(NAN));
    T mu_neg = -R.pmu / (1.0 - R.pmu);
    T upq = R.sqrt_up * R.sqrt_up;
    if (R.vortical) { R.qC = 1.0 / (1.0 - R.um); R.qn = (upq - R.um) / (1.0 - R.um); }
    else { R.qC = T(1.0); R.qn = upq; }
    R.sqrt_eps = sqrt(fmax(1.0 - R.qn, T(0.0)));
    R.gc = 1.0 / sqrt(1.0 - mu_neg);
    R.mp = mu_neg / (1.0 - mu_neg);
    R.K2 = 2.0 * ellip_k(R.pmu) / R.pscale;
    R.vabsalpha = fabs(alpha); R.valpha2 = alpha * alpha; R.vabsbeta = fabs(beta) + kEps;
    return R;
}

KS_HD int anchor_interval(int M, double one_minus_k) {
    double scaled = M * sqrt(fmax(one_minus_k, 0.0) / 2e-5);
    double v = fmin(scaled, double(M));
    int t = int(v);
    return t < 4 ? 4 : (t > M ? M : t);
}

}  // namespace ks
