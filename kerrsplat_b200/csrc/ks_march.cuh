// ks_march.cuh -- the fused Recurrence(M) march of one ray (quadrature.jl:231-296) in precision T,
// reading the FP64 plan and anchor table built by regenerate.
//
// T = double is the plain FP64 port of the reference's march_ray, sample for sample. T = float is
// the mixed path: the smooth integrands, the interval increments (their logarithms and the polar
// closed form) and the sample positions run in FP32, reset to the FP64 anchors every M samples; the
// smooth t-integrand uses the cancellation-free large-r form there (its r^2 terms would otherwise lose
// everything in FP32 at r ~ 1e4). The Jacobi states of both recurrences, r, cos theta, the visibility
// test and the t~/phi running sums stay in FP64 (GeoT), a few multiplications and one division per
// half step:
// - the visibility test is krang_visible (recurrence.jl:299-308), whose boundary |beta| =
//   beta_boundary(theta_s) is the polar turning point itself, so the samples next to a turning point
//   flip validity under an FP32 cos theta (2.5e-4 of the configuration-2 image came from those flags);
// - FP32 recurrences drift between anchors (6e-4 on a 16^2, N = 128 scene at M = 64, falling as the
//   anchor spacing shrinks).
#pragma once
#include "ks_plan.cuh"

namespace ks {

template <class T>
struct Sample {
    T t, r, theta, cos_theta, phi;
    bool nur, nutheta, ok;
};

// The type of Mino times: FP64 for the FP32 and FP64 marches (sample times compared in FP64), the
// dual itself when the times carry derivatives (the spacetime duals: tau_k = k tau_total / (N + 1)).
template <class T> struct TimeOf { using type = double; };
template <class S, int N> struct TimeOf<Dual<S, N>> { using type = Dual<S, N>; };
template <class T> using TimeT = typename TimeOf<T>::type;

// The precision of the geometry state (the Jacobi states, r, cos theta, the visibility test and the
// running sums): FP64 under the FP32 march, the march's own type otherwise.
template <class T> struct GeoOf { using type = T; };
template <> struct GeoOf<float> { using type = double; };
template <class T> using GeoT = typename GeoOf<T>::type;

template <class T>
struct MarchRay {
    using PT = GeoT<T>;
    int rcase;
    PT k, m0, m1, m2, m3;
    T c, fo;
    TimeT<T> tau_valid, dtau, fo_d;  // compared against sample times in FP64
    PT pmu, pscale, sqrt_up, um, up_m_um, psign;
    T tempfac, poffset;
    bool vortical, scattering;
    T a, lam, eta, rp, rmn, sp, sm, Qt, Qtm, Qphi, Qphim, r4, qC, qn, sqrt_eps, gc, mp, K2;
    PT vabsalpha, valpha2, vabsbeta, vabscos, vcos2, pa;   // krang_visible's constants (pa: the spin)
    JS<PT> dr, dth;
    int turn_k, Manchor, nanch, nsamp;
    long long anchor_off;
};

struct PlanView {
    const double* f;       // PF_COUNT arrays of stride npad
    long long npad;
    const double* anchors; // AF_COUNT doubles per anchor
    const long long* anchor_off;
    __device__ __forceinline__ double get(int field, long long j) const { return f[field * npad + j]; }
};

template <class T>
__device__ __forceinline__ MarchRay<T> load_ray(const PlanView& P, const Spacetime& st, long long j) {
    MarchRay<T> R;
    R.rcase = int(P.get(PF_CASE, j));
    using PT = GeoT<T>;
    R.k = PT(P.get(PF_K, j)); R.c = T(P.get(PF_C, j)); R.fo = T(P.get(PF_FO, j));
    R.m0 = PT(P.get(PF_MAP0, j)); R.m1 = PT(P.get(PF_MAP1, j)); R.m2 = PT(P.get(PF_MAP2, j)); R.m3 = PT(P.get(PF_MAP3, j));
    R.tau_valid = P.get(PF_TAU_VALID, j); R.dtau = P.get(PF_DTAU, j); R.fo_d = P.get(PF_FO, j);
    R.pmu = PT(P.get(PF_PMU, j)); R.pscale = PT(P.get(PF_PSCALE, j)); R.tempfac = T(P.get(PF_TEMPFAC, j));
    R.poffset = T(P.get(PF_POFFSET, j)); R.sqrt_up = PT(P.get(PF_SQRTUP, j)); R.um = PT(P.get(PF_UM, j));
    R.up_m_um = PT(P.get(PF_UPMUM, j)); R.psign = PT(P.get(PF_PSIGN, j));
    R.vortical = P.get(PF_VORTICAL, j) != 0.0; R.scattering = P.get(PF_SCATTER, j) != 0.0;
    R.a = T(st.a); R.lam = T(P.get(PF_LAM, j)); R.eta = T(P.get(PF_ETA, j)); R.rp = T(st.rp); R.rmn = T(st.rmn);
    R.sp = T(P.get(PF_SP, j)); R.sm = T(P.get(PF_SM, j)); R.Qt = T(P.get(PF_QT, j)); R.Qtm = T(P.get(PF_QTM, j));
    R.Qphi = T(P.get(PF_QPHI, j)); R.Qphim = T(P.get(PF_QPHIM, j)); R.r4 = T(P.get(PF_R4, j));
    R.qC = T(P.get(PF_QC, j)); R.qn = T(P.get(PF_QN, j)); R.sqrt_eps = T(P.get(PF_SQRTEPS, j));
    R.gc = T(P.get(PF_GC, j)); R.mp = T(P.get(PF_MP, j)); R.K2 = T(P.get(PF_K2, j));
    R.vabsalpha = PT(P.get(PF_VABSALPHA, j)); R.valpha2 = PT(P.get(PF_VALPHA2, j)); R.vabsbeta = PT(P.get(PF_VABSBETA, j));
    R.vabscos = PT(st.abscos); R.vcos2 = PT(st.cos2); R.pa = PT(st.a);
    R.dr = {PT(P.get(PF_DR_SN, j)), PT(P.get(PF_DR_CN, j)), PT(P.get(PF_DR_DN, j))};
    R.dth = {PT(P.get(PF_DTH_SN, j)), PT(P.get(PF_DTH_CN, j)), PT(P.get(PF_DTH_DN, j))};
    R.turn_k = int(P.get(PF_TURN_K, j));
    R.Manchor = int(P.get(PF_MANCHOR, j));
    R.nanch = int(P.get(PF_NANCH, j));
    R.nsamp = int(P.get(PF_NSAMP, j));
    R.anchor_off = P.anchor_off[j];
    return R;
}

// ---- per-sample geometry (recurrence.jl:169-308, quadrature.jl:110-215) ---------------------------

template <class T> __device__ __forceinline__ T kpi() { return T(kPi); }
template <> __device__ __forceinline__ double kpi<double>() { return kPi; }
template <> __device__ __forceinline__ float kpi<float>() { return 3.14159265358979323846f; }
template <class T> __device__ __forceinline__ T keps() { return T(kEps); }
template <> __device__ __forceinline__ double keps<double>() { return kEps; }
template <> __device__ __forceinline__ float keps<float>() { return 1.1920929e-7f; }

template <class T>
__device__ __forceinline__ GeoT<T> radius(const MarchRay<T>& R, const JS<GeoT<T>>& x) {
    using PT = GeoT<T>;
    if (R.rcase == 2) {
        PT cn2 = R.m2 * x.cn * x.cn;
        return (R.m1 * cn2 - R.m0 * R.m3) / (cn2 - R.m3);
    } else if (R.rcase == 3) {
        return (R.m0 + R.m1 * x.cn) / (R.m2 + R.m3 * x.cn);
    }
    PT sc = x.sn / x.cn;
    return -(R.m0 * (R.m2 - sc) / (PT(1) + R.m2 * sc) + R.m1);
}

// cos theta in the polar precision (and theta in the march's, from the rounded cos theta)
template <class T>
__device__ __forceinline__ void polar_cos(const MarchRay<T>& R, const JS<GeoT<T>>& x, T& theta, GeoT<T>& cth, bool& nu) {
    using PT = GeoT<T>;
    PT snX = x.sn / (R.pscale * x.dn);
    PT c;
    if (R.vortical) {
        c = R.psign * sqrt(fmax(R.um + R.up_m_um * snX * snX, PT(0)));
        nu = R.psign * x.sn * x.cn > PT(0);
    } else {
        c = R.psign * R.sqrt_up * snX;
        nu = R.psign * x.cn > PT(0);
    }
    c = fmin(PT(1), fmax(PT(-1), c));
    cth = c;
    theta = acos(T(c));
}

template <class T>
__device__ __forceinline__ bool visible(const MarchRay<T>& R, GeoT<T> cths) {
    using PT = GeoT<T>;
    if (!(cths > R.vabscos)) return true;
    PT c2 = cths * cths;
    PT s2 = PT(1) - c2;
    PT amin = R.pa * sqrt(s2);
    if (!(R.vabsalpha >= amin + keps<PT>())) return true;
    PT temp = (R.vcos2 - c2) * (R.valpha2 - R.pa * R.pa * s2) / (c2 - PT(1));
    PT bb = sqrt(fmax(temp, PT(0)));
    return !(R.vabsbeta < bb);
}

template <class T>
struct Point {
    T r, theta, cth, s, sn, cn, gt, gphi;
    GeoT<T> cthp;   // cos theta in the polar precision (the visibility test)
    bool nur, nuth;
};

// sn, cn of the polar map and 1/dn (the smooth integrand's inputs) in the march's precision
template <class T>
__device__ __forceinline__ void polar_map(const MarchRay<T>& R, const JS<GeoT<T>>& xt, Point<T>& p, T& dn_inv) {
    if constexpr (std::is_same<T, GeoT<T>>::value) {
        p.sn = xt.sn / (R.pscale * xt.dn);
        p.cn = xt.cn / xt.dn;
        dn_inv = T(1) / xt.dn;
    } else {
        const T sn = T(xt.sn), cn = T(xt.cn), dn = T(xt.dn);
        dn_inv = T(1) / dn;
        p.sn = sn * dn_inv / T(R.pscale);
        p.cn = cn * dn_inv;
    }
}

template <class T>
__device__ __forceinline__ void smooth(const MarchRay<T>& R, Point<T>& p, T dn) {
    const T a = R.a, lam = R.lam, r = p.r, s = p.s;
    T D = r * r - T(2) * r + a * a;
    T s2 = T(1) - p.cth * p.cth;
    T wp = s * R.rp / (r * (r - R.rp)) / R.sp;
    T wm = s * R.rmn / (r * (r - R.rmn)) / R.sm;
    T P = r * r + a * a - a * lam;
    if constexpr (is_f32<T>) {
        if (r > T(64) && P > T(0)) {
            // dt/dtau - |s|(1 + 2/r) without cancellation (see the anchor integrand)
            T Qv = R.eta + (lam - a) * (lam - a);
            T as = fabs(s);
            T diff = D * Qv / (P + as) * (T(1) + T(2) / r) + T(2) * (T(2) * r - a * a) * P / (r * D);
            p.gt = diff + a * (lam - a * s2) - R.Qt * wp - R.Qtm * wm;
        } else {
            T ft = (r * r + a * a) * P / D + a * (lam - a * s2);
            p.gt = ft - fabs(s) * (T(1) + T(2) / r) - R.Qt * wp - R.Qtm * wm;
        }
    } else {
        T ft = (r * r + a * a) * (r * r + a * a - a * lam) / D + a * (lam - a * s2);
        p.gt = ft - fabs(s) * (T(1) + T(2) / r) - R.Qt * wp - R.Qtm * wm;
    }
    T fphi = a * (T(2) * r - a * lam) / D;
    T gpol = lam * R.qC * (T(1) - R.gc * dn * (T(1) - R.mp * p.cn * p.cn / T(2))) / (T(1) - R.qn * p.sn * p.sn);
    p.gphi = fphi - R.Qphi * wp - R.Qphim * wm + gpol;
}

template <class T>
__device__ __forceinline__ T r_pot(const MarchRay<T>& R, T r) {
    T P = r * r + R.a * R.a - R.a * R.lam;
    T D = r * r - T(2) * r + R.a * R.a;
    return P * P - D * (R.eta + (R.lam - R.a) * (R.lam - R.a));
}

template <class T>
__device__ __forceinline__ Point<T> ray_point(const MarchRay<T>& R, const JS<GeoT<T>>& xr, const JS<GeoT<T>>& xt, TimeT<T> tau) {
    Point<T> p;
    p.r = T(radius(R, xr));
    polar_cos(R, xt, p.theta, p.cthp, p.nuth);
    p.cth = T(p.cthp);
    p.nur = tau < R.fo_d;
    p.s = (p.nur ? T(-1) : T(1)) * sqrt(fmax(r_pot(R, p.r), T(0)));
    T dn_inv;
    polar_map(R, xt, p, dn_inv);
    smooth(R, p, dn_inv);
    return p;
}

template <class T>
__device__ __forceinline__ Point<T> turning_point(const MarchRay<T>& R, const JS<GeoT<T>>& xt) {
    Point<T> p;
    p.r = R.r4;
    polar_cos(R, xt, p.theta, p.cthp, p.nuth);
    p.cth = T(p.cthp);
    p.nur = true;
    p.s = T(0);
    T dn_inv;
    polar_map(R, xt, p, dn_inv);
    smooth(R, p, dn_inv);
    return p;
}

template <class T>
__device__ __forceinline__ T polar_closed(const MarchRay<T>& R, TimeT<T> tau, T sn, T cn) {
    T X = (T(tau) + R.poffset) / R.tempfac;
    T nw = floor((X + R.K2 / T(2)) / R.K2);
    T A = (atan(R.sqrt_eps * sn / cn) + nw * kpi<T>()) / R.sqrt_eps;
    T ph = atan(sn / cn) + nw * kpi<T>();
    T e = R.sqrt_eps * R.sqrt_eps;
    return R.lam * R.qC * R.tempfac * R.gc * ((T(1) + R.mp * e / (T(2) * R.qn)) * A - R.mp / (T(2) * R.qn) * ph);
}

// Interval increment (quadrature.jl:205-215); pca = polar_closed at the interval's start, carried
// from the previous interval (the same inputs, hence the same value).
template <class T>
__device__ __forceinline__ void increment(const MarchRay<T>& R, const Point<T>& pa, const Point<T>& pm, const Point<T>& pb,
                                          TimeT<T> ta, TimeT<T> tb, T pca, T pcb, T& It, T& Iphi) {
    T h = T(tb - ta);
    T ra = pa.r, rb = pb.r;
    T dFr = (rb - ra) + T(2) * log(rb / ra);
    T dFp = log((rb - R.rp) * ra / ((ra - R.rp) * rb)) / R.sp;
    T dFm = log((rb - R.rmn) * ra / ((ra - R.rmn) * rb)) / R.sm;
    It = h / T(6) * (pa.gt + T(4) * pm.gt + pb.gt) + fabs(dFr) + R.Qt * dFp + R.Qtm * dFm;
    Iphi = h / T(6) * (pa.gphi + T(4) * pm.gphi + pb.gphi) + R.Qphi * dFp + R.Qphim * dFm + pcb - pca;
}

template <class T>
__device__ __forceinline__ JS<T> load_js(const double* rec, int off) {
    return {T(rec[off]), T(rec[off + 1]), T(rec[off + 2])};
}

// March samples [k_begin, k_end) of ray j and call f(k, sample) for each (quadrature.jl:231-296): the
// march starts at the last anchor at or before k_begin (its Jacobi states, t~ and phi from the table)
// and runs silently up to k_begin, so the lanes of a warp call f the same number of times whatever
// their anchor spacing. At every anchor the quadrature's t~ and phi are replaced by the anchor's; with
// RESID the largest |quadrature - anchor| of the ray (cache.residual_t / residual_phi) is tracked.
template <bool RESID, class T, class F>
__device__ __forceinline__ void march_impl(const PlanView& P, long long j, const MarchRay<T>& R, F& f, int k_begin, int k_end,
                                           double& resid_t, double& resid_phi) {
    double rt = 0.0, rphi = 0.0;
    if (k_end > R.nsamp + 1) k_end = R.nsamp + 1;
    if (k_begin < k_end) {
        const double dtau = R.dtau;
        const double h = dtau / 2.0;
        int m = (k_begin - 1) / R.Manchor;
        if (m > R.nanch - 1) m = R.nanch - 1;
        const int ka = 1 + m * R.Manchor;
        const double* A0 = P.anchors + (R.anchor_off + m) * AF_COUNT;
        using PT = GeoT<T>;
        JS<PT> xr = load_js<PT>(A0, AF_XR_SN);
        JS<PT> xt = load_js<PT>(A0, AF_XT_SN);
        Point<T> pa = ray_point(R, xr, xt, ka * dtau);
        T pca = polar_closed(R, ka * dtau, pa.sn, pa.cn);
        PT t = PT(A0[AF_T]), phi = PT(A0[AF_PHI]);
        if (ka >= k_begin) {
            Sample<T> s{T(t), pa.r, pa.theta, pa.cth, T(phi), pa.nur, pa.nuth, (ka * dtau <= R.tau_valid) && visible(R, pa.cthp)};
            f(ka, s);
        }
        int next_anchor = ka + R.Manchor;
        ++m;
        for (int k = ka + 1; k < k_end; ++k) {
            double ta = (k - 1) * dtau, tb = k * dtau;
            xr = jstep(xr, R.dr, R.k);
            xt = jstep(xt, R.dth, R.pmu);
            Point<T> pm = ray_point(R, xr, xt, ta + h);
            const bool anchor = (k == next_anchor);
            const double* Am = P.anchors + (R.anchor_off + m) * AF_COUNT;
            if (anchor) {
                xr = load_js<PT>(Am, AF_XR_SN); xt = load_js<PT>(Am, AF_XT_SN);
            } else {
                xr = jstep(xr, R.dr, R.k);
                xt = jstep(xt, R.dth, R.pmu);
            }
            Point<T> pb = ray_point(R, xr, xt, tb);
            T pcb = polar_closed(R, tb, pb.sn, pb.cn);
            if (k == R.turn_k) {
                const double* pf = P.f;
                const long long np = P.npad;
                JS<PT> p1r = {PT(pf[PF_P1R_SN * np + j]), PT(pf[PF_P1R_CN * np + j]), PT(pf[PF_P1R_DN * np + j])};
                JS<PT> p1t = {PT(pf[PF_P1T_SN * np + j]), PT(pf[PF_P1T_CN * np + j]), PT(pf[PF_P1T_DN * np + j])};
                JS<PT> p2r = {PT(pf[PF_P2R_SN * np + j]), PT(pf[PF_P2R_CN * np + j]), PT(pf[PF_P2R_DN * np + j])};
                JS<PT> p2t = {PT(pf[PF_P2T_SN * np + j]), PT(pf[PF_P2T_CN * np + j]), PT(pf[PF_P2T_DN * np + j])};
                JS<PT> ptt = {PT(pf[PF_PTT_SN * np + j]), PT(pf[PF_PTT_CN * np + j]), PT(pf[PF_PTT_DN * np + j])};
                double fo = R.fo_d;
                Point<T> pt = turning_point(R, ptt);
                Point<T> p1 = ray_point(R, p1r, p1t, (ta + fo) / 2.0);
                Point<T> p2 = ray_point(R, p2r, p2t, (fo + tb) / 2.0);
                T pct = polar_closed(R, fo, pt.sn, pt.cn);
                T It1, Ip1, It2, Ip2;
                increment(R, pa, p1, pt, ta, fo, pca, pct, It1, Ip1);
                increment(R, pt, p2, pb, fo, tb, pct, pcb, It2, Ip2);
                t += PT(It1) + PT(It2); phi += PT(Ip1) + PT(Ip2);
            } else {
                T It, Ip;
                increment(R, pa, pm, pb, ta, tb, pca, pcb, It, Ip);
                t += PT(It); phi += PT(Ip);
            }
            if (anchor) {
                if (Am[AF_OK] != 0.0) {
                    const double at = Am[AF_T], ap = Am[AF_PHI];
                    if constexpr (RESID) {
                        rt = fmax(rt, fabs(double(t) - at));
                        rphi = fmax(rphi, fabs(double(phi) - ap));
                    }
                    t = PT(at); phi = PT(ap);
                }
                ++m;
                next_anchor += R.Manchor;
            }
            if (k >= k_begin) {
                Sample<T> s{T(t), pb.r, pb.theta, pb.cth, T(phi), pb.nur, pb.nuth, (tb <= R.tau_valid) && visible(R, pb.cthp)};
                f(k, s);
            }
            pa = pb;
            pca = pcb;
        }
    }
    resid_t = rt;
    resid_phi = rphi;
}

// March ray j with its N samples and call f(k, sample) for k = 1..N; returns the largest anchor residuals.
template <class T, class F>
__device__ __forceinline__ void march(const PlanView& P, const Spacetime& st, long long j, const MarchRay<T>& R,
                                      F& f, double& resid_t, double& resid_phi) {
    (void)st;
    march_impl<true>(P, j, R, f, 1, R.nsamp + 1, resid_t, resid_phi);
}

// March samples [k_begin, k_end) of ray j (no residuals): the work segments of the sample stream.
template <class T, class F>
__device__ __forceinline__ void march_range(const PlanView& P, long long j, const MarchRay<T>& R, F& f, int k_begin, int k_end) {
    double rt, rp;
    march_impl<false>(P, j, R, f, k_begin, k_end, rt, rp);
}

}  // namespace ks
