// ks_lib.cu -- libkerrsplat_b200.so: the kernels of the render hot path and the C ABI of
// include/kerrsplat_b200.h.
//
// Pipeline of one context (the device-side GeodesicCache of cache.jl:85-125):
//   ks_regenerate: k_root_case (K0, screen order) -> stable radix sort by root case (4, 2, 0 real
//     roots; cub, deterministic) -> k_build_plan (K1: FP64 per-ray constants, sorted order) ->
//     exclusive scan of anchor counts -> k_anchor_segments (one thread per (ray, anchor): Jacobi
//     states, validity, closed-form parts and the Gauss-Legendre integral of the smooth part since
//     the previous anchor) -> k_anchor_prefix (per-ray running sums).
//   ks_thin_image / ks_render: k_splat_table (per-splat FP64 constants) -> k_thin / k_polarized
//     (one thread per ray, the fused march with the consumer folded over the samples) -> k_unsort.
#include <cub/cub.cuh>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/kerrsplat_b200.h"
#include "ks_dft.cuh"
#include "ks_transfer.cuh"

using namespace ks;

__constant__ MomentCoeffs c_moments;

namespace {

constexpr int kBlock = 128;

// ---- kernels: regenerate ---------------------------------------------------------------------------

__global__ void k_root_case(Spacetime st, const double* __restrict__ alpha, const double* __restrict__ beta, long long npix,
                            unsigned char* __restrict__ key, long long* __restrict__ idx) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= npix) return;
    RayC R = build_ray(st, alpha[i], beta[i]);
    key[i] = (unsigned char)(4 - R.numreals);   // 4 real roots first (pixel_constants.jl:167-176)
    idx[i] = i;
}

template <class T>
__device__ __forceinline__ MarchRay<T> march_ray_of(const RayCT<T>& R, const SpacetimeT<T>& st, TimeT<T> dtau) {
    MarchRay<T> M;
    M.rcase = R.rcase; M.k = R.k; M.c = R.c; M.fo = R.fo; M.fo_d = R.fo;
    M.m0 = R.map[0]; M.m1 = R.map[1]; M.m2 = R.map[2]; M.m3 = R.map[3];
    M.tau_valid = R.tau_valid; M.dtau = dtau;
    M.pmu = R.pmu; M.pscale = R.pscale; M.tempfac = R.tempfac; M.poffset = R.poffset; M.sqrt_up = R.sqrt_up;
    M.um = R.um; M.up_m_um = R.up_m_um; M.psign = R.psign; M.vortical = R.vortical; M.scattering = R.scattering;
    M.a = st.a; M.lam = R.lam; M.eta = R.eta; M.rp = st.rp; M.rmn = st.rmn; M.sp = R.sp; M.sm = R.sm;
    M.Qt = R.Qt; M.Qtm = R.Qtm; M.Qphi = R.Qphi; M.Qphim = R.Qphim; M.r4 = R.r4; M.qC = R.qC; M.qn = R.qn;
    M.sqrt_eps = R.sqrt_eps; M.gc = R.gc; M.mp = R.mp; M.K2 = R.K2;
    M.vabsalpha = R.vabsalpha; M.valpha2 = R.valpha2; M.vabsbeta = R.vabsbeta; M.vabscos = st.abscos; M.vcos2 = st.cos2;
    M.pa = st.a;
    return M;
}

template <class T>
__device__ __forceinline__ JS<T> xr_at(const RayCT<T>& R, TimeT<T> tau) { return jstate(R.c * (R.fo - tau), R.k); }
template <class T>
__device__ __forceinline__ JS<T> xt_at(const RayCT<T>& R, TimeT<T> tau) { return jstate(R.pscale * (tau + R.poffset) / R.tempfac, R.pmu); }

__global__ void k_build_plan(Spacetime st, const double* __restrict__ alpha, const double* __restrict__ beta,
                             const long long* __restrict__ perm, long long npix, long long npad, double* __restrict__ f,
                             long long* __restrict__ nanch_out) {
    long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= npix) return;
    long long i = perm[j];
    RayC R = build_ray(st, alpha[i], beta[i]);
    auto put = [&](int field, double v) { f[field * npad + j] = v; };
    int Nj = st.N;
    if (st.density > 0.0) {
        const double want = 64.0 * ceil(st.density * R.tau_total / 64.0);
        Nj = (want > 0.0) ? int(fmin(double(st.N), fmax(double(st.nmin), want))) : st.nmin;
    }
    double dtau = R.tau_total / (Nj + 1);
    double h = dtau / 2.0;
    int Man = anchor_interval(st.M, 1.0 - R.k);
    int nanch = (Nj - 1) / Man + 1;
    put(PF_NSAMP, Nj);
    put(PF_ALPHA, R.alpha); put(PF_BETA, R.beta); put(PF_ETA, R.eta); put(PF_LAM, R.lam);
    put(PF_NUMREALS, R.numreals); put(PF_CASE, R.rcase);
    put(PF_K, R.k); put(PF_C, R.c); put(PF_FO, R.fo);
    put(PF_MAP0, R.map[0]); put(PF_MAP1, R.map[1]); put(PF_MAP2, R.map[2]); put(PF_MAP3, R.map[3]);
    put(PF_TAU_VALID, R.tau_valid); put(PF_TAU_TOTAL, R.tau_total); put(PF_DTAU, dtau);
    put(PF_PMU, R.pmu); put(PF_PSCALE, R.pscale); put(PF_TEMPFAC, R.tempfac); put(PF_POFFSET, R.poffset);
    put(PF_SQRTUP, R.sqrt_up); put(PF_UM, R.um); put(PF_UPMUM, R.up_m_um); put(PF_PSIGN, R.psign);
    put(PF_VORTICAL, R.vortical ? 1.0 : 0.0); put(PF_GTHO, R.gtho);
    put(PF_SP, R.sp); put(PF_SM, R.sm); put(PF_QT, R.Qt); put(PF_QTM, R.Qtm); put(PF_QPHI, R.Qphi); put(PF_QPHIM, R.Qphim);
    put(PF_R4, R.r4); put(PF_SCATTER, R.scattering ? 1.0 : 0.0);
    put(PF_QC, R.qC); put(PF_QN, R.qn); put(PF_SQRTEPS, R.sqrt_eps); put(PF_GC, R.gc); put(PF_MP, R.mp); put(PF_K2, R.K2);
    put(PF_VABSALPHA, R.vabsalpha); put(PF_VALPHA2, R.valpha2); put(PF_VABSBETA, R.vabsbeta);
    JS<double> dr = jstep_constants(-R.c * h, R.k);
    JS<double> dth = jstep_constants(R.pscale * h / R.tempfac, R.pmu);
    put(PF_DR_SN, dr.sn); put(PF_DR_CN, dr.cn); put(PF_DR_DN, dr.dn);
    put(PF_DTH_SN, dth.sn); put(PF_DTH_CN, dth.cn); put(PF_DTH_DN, dth.dn);
    // the interval that holds the radial turning point of a scattering ray (quadrature.jl:269)
    int turn_k = -1;
    if (R.scattering) {
        for (int k = 2; k <= Nj; ++k) {
            double ta = (k - 1) * dtau, tb = k * dtau;
            if (ta < R.fo && R.fo < tb) { turn_k = k; break; }
        }
    }
    put(PF_TURN_K, turn_k);
    if (turn_k > 0) {
        double ta = (turn_k - 1) * dtau, tb = turn_k * dtau;
        JS<double> a1 = xr_at(R, (ta + R.fo) / 2.0), b1 = xt_at(R, (ta + R.fo) / 2.0);
        JS<double> a2 = xr_at(R, (R.fo + tb) / 2.0), b2 = xt_at(R, (R.fo + tb) / 2.0);
        JS<double> pt = xt_at(R, R.fo);
        put(PF_P1R_SN, a1.sn); put(PF_P1R_CN, a1.cn); put(PF_P1R_DN, a1.dn);
        put(PF_P1T_SN, b1.sn); put(PF_P1T_CN, b1.cn); put(PF_P1T_DN, b1.dn);
        put(PF_P2R_SN, a2.sn); put(PF_P2R_CN, a2.cn); put(PF_P2R_DN, a2.dn);
        put(PF_P2T_SN, b2.sn); put(PF_P2T_CN, b2.cn); put(PF_P2T_DN, b2.dn);
        put(PF_PTT_SN, pt.sn); put(PF_PTT_CN, pt.cn); put(PF_PTT_DN, pt.dn);
    } else {
        for (int q = PF_P1R_SN; q <= PF_PTT_DN; ++q) put(q, 0.0);
    }
    put(PF_MANCHOR, Man); put(PF_NANCH, nanch);
    put(PF_R1RE, R.rre[0]); put(PF_R1IM, R.rim[0]); put(PF_R2RE, R.rre[1]); put(PF_R2IM, R.rim[1]);
    put(PF_R3RE, R.rre[2]); put(PF_R3IM, R.rim[2]); put(PF_R4RE, R.rre[3]); put(PF_R4IM, R.rim[3]);
    nanch_out[j] = nanch;
}

// The smooth integrands at tau from direct Jacobi states, the t part in its large-r form past r = 64.
template <class T>
__device__ __forceinline__ void anchor_integrand(const RayCT<T>& R, const MarchRay<T>& M, TimeT<T> tau, T& gt, T& gp) {
    JS<T> xr = xr_at(R, tau), xt = xt_at(R, tau);
    Point<T> p = ray_point(M, xr, xt, tau);
    gt = p.gt; gp = p.gphi;
    T r = p.r, a = M.a, lam = M.lam;
    T P = r * r + a * a - a * lam;
    if (r > 64.0 && P > 0.0) {
        T D = r * r - 2.0 * r + a * a;
        T Qv = M.eta + (lam - a) * (lam - a);
        T as = fabs(p.s);
        T diff = D * Qv / (P + as) * (1.0 + 2.0 / r) + 2.0 * (2.0 * r - a * a) * P / (r * D);
        T s2 = 1.0 - p.cth * p.cth;
        T wp = p.s * M.rp / (r * (r - M.rp)) / M.sp;
        T wm = p.s * M.rmn / (r * (r - M.rmn)) / M.sm;
        gt = diff + a * (lam - a * s2) - M.Qt * wp - M.Qtm * wm;
    }
}

__constant__ double c_gl_x[16];
__constant__ double c_gl_w[16];

template <class T>
__device__ void gl_panel(const RayCT<T>& R, const MarchRay<T>& M, TimeT<T> ta, TimeT<T> tb, T& It, T& Ip) {
    const TimeT<T> mid = 0.5 * (ta + tb), half = 0.5 * (tb - ta);
    T st = T(0.0), sp = T(0.0);
    for (int i = 0; i < 16; ++i) {
        T gt, gp;
        anchor_integrand(R, M, mid + half * c_gl_x[i], gt, gp);
        st += c_gl_w[i] * gt; sp += c_gl_w[i] * gp;
    }
    It = half * st; Ip = half * sp;
}

constexpr int kAnchorPanelSamples = 4;

__global__ void k_anchor_segments(Spacetime st, const double* __restrict__ alpha, const double* __restrict__ beta,
                                  const long long* __restrict__ perm, long long npix, long long npad, const double* __restrict__ f,
                                  const long long* __restrict__ aoff, double* __restrict__ anchors) {
    long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    int m = blockIdx.y;
    if (j >= npix) return;
    int nanch = int(f[PF_NANCH * npad + j]);
    if (m >= nanch) return;
    long long i = perm[j];
    RayC R = build_ray(st, alpha[i], beta[i]);
    int Man = int(f[PF_MANCHOR * npad + j]);
    double dtau = f[PF_DTAU * npad + j];
    MarchRay<double> M = march_ray_of(R, st, dtau);
    int k = 1 + m * Man;
    double tau = k * dtau;
    double* A = anchors + (aoff[j] + m) * AF_COUNT;
    JS<double> xr = xr_at(R, tau), xt = xt_at(R, tau);
    A[AF_XR_SN] = xr.sn; A[AF_XR_CN] = xr.cn; A[AF_XR_DN] = xr.dn;
    A[AF_XT_SN] = xt.sn; A[AF_XT_CN] = xt.cn; A[AF_XT_DN] = xt.dn;
    double th, cth; bool nu;
    polar_cos(M, xt, th, cth, nu);
    bool ok = (tau <= R.tau_valid) && visible(M, cth);
    A[AF_OK] = ok ? 1.0 : 0.0;
    A[AF_PAD] = 0.0;
    if (!(tau <= R.tau_valid)) {
        A[AF_T] = 0.0; A[AF_PHI] = 0.0; A[AF_SEG_T] = 0.0; A[AF_SEG_PHI] = 0.0;
        return;
    }
    // closed-form parts at tau, accumulated from the observer
    Point<double> p = ray_point(M, xr, xt, tau);
    double r = p.r;
    double F = r + 2.0 * log(r);
    double L = (R.scattering && tau > R.fo) ? F - 2.0 * (R.r4 + 2.0 * log(R.r4)) : -F;
    double lp = log((r - st.rp) / r) / R.sp;
    double lm = log((r - st.rmn) / r) / R.sm;
    JS<double> x0 = xt_at(R, 0.0);
    double sn0 = x0.sn / (R.pscale * x0.dn), cn0 = x0.cn / x0.dn;
    A[AF_T] = L + R.Qt * lp + R.Qtm * lm;
    A[AF_PHI] = R.Qphi * lp + R.Qphim * lm + polar_closed(M, tau, p.sn, p.cn) - polar_closed(M, 0.0, sn0, cn0);
    // smooth part over (previous anchor, tau]
    double ta = (m == 0) ? 0.0 : (1 + (m - 1) * Man) * dtau;
    int nsamp = (m == 0) ? 1 : Man;
    int np = (m == 0) ? 1 : (nsamp + kAnchorPanelSamples - 1) / kAnchorPanelSamples;
    double hp = (tau - ta) / np;
    double It = 0.0, Ip = 0.0;
    for (int q = 0; q < np; ++q) {
        double a0 = ta + q * hp, b0 = (q == np - 1) ? tau : ta + (q + 1) * hp;
        double t1, p1;
        if (R.scattering && a0 < R.fo && R.fo < b0) {
            gl_panel(R, M, a0, R.fo, t1, p1); It += t1; Ip += p1;
            gl_panel(R, M, R.fo, b0, t1, p1); It += t1; Ip += p1;
        } else {
            gl_panel(R, M, a0, b0, t1, p1); It += t1; Ip += p1;
        }
    }
    A[AF_SEG_T] = It; A[AF_SEG_PHI] = Ip;
}

__global__ void k_anchor_prefix(long long npix, long long npad, const double* __restrict__ f, const long long* __restrict__ aoff,
                                double* __restrict__ anchors) {
    long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= npix) return;
    int nanch = int(f[PF_NANCH * npad + j]);
    double st = 0.0, sp = 0.0;
    for (int m = 0; m < nanch; ++m) {
        double* A = anchors + (aoff[j] + m) * AF_COUNT;
        st += A[AF_SEG_T]; sp += A[AF_SEG_PHI];
        A[AF_T] += st; A[AF_PHI] += sp;
    }
}

// ---- kernels: splat tables ---------------------------------------------------------------------------

// the table (and knot array) in FP32 for the mixed kernels' staging copy, zero-padded to np4 floats
__global__ void k_tab_f32(long long n, long long np4, const double* __restrict__ src, float* __restrict__ dst) {
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q < np4) dst[q] = q < n ? float(src[q]) : 0.f;
}

// K0 and K1 from K_nu(x) = int_0^inf exp(-x cosh t) cosh(nu t) dt by the trapezoidal rule.
__host__ __device__ void besselk01(double x, double& k0, double& k1) {
    // trapezoid in t on exp(-x (cosh t - 1)) (the factor exp(-x) applied at the end); the step
    // resolves the Gaussian core of width 1/sqrt(x) (error ~ exp(-2 pi^2 / (x h^2)) < 1e-17)
    const double h = fmin(0.125, 0.6 / sqrt(x));
    double s0 = 0.5, s1 = 0.5;
    for (int j = 1; j < 20000; ++j) {
        double t = j * h;
        double ch = cosh(t);
        double e = exp(-x * (ch - 1.0));
        s0 += e;
        s1 += e * ch;
        if (e < 1e-18 * s0) break;
    }
    double ex = exp(-x);
    k0 = h * s0 * ex; k1 = h * s1 * ex;
}

struct SetDesc {
    int kind, nrows, nsplat, first;   // first = index of its first splat in the concatenated table
    const double* params;
    const double* hyp;
    double gmax;
    int koff, nk;                     // knot splats: offset of the set's first knot record, knot count
    const double* knots;              // the knot array (device)
};

__global__ void k_splat_table(SetDesc d, double* __restrict__ tab) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.nsplat) return;
    const double* p = d.params + (long long)d.nrows * i;
    double* o = tab + (long long)(d.first + i) * ST_COUNT;
    for (int q = 0; q < ST_COUNT; ++q) o[q] = 0.0;
    o[ST_KIND] = d.kind;
    o[ST_CX] = p[0]; o[ST_CY] = p[1]; o[ST_CZ] = p[2];
    o[ST_T0] = p[10]; o[ST_OMEGA] = p[d.nrows - 1];
    o[ST_ES1] = exp(-p[3]); o[ST_ES2] = exp(-p[4]); o[ST_ES3] = exp(-p[5]);
    double q1 = p[6], q2 = p[7], q3 = p[8], q4 = p[9];
    double n = sqrt(q1 * q1 + q2 * q2 + q3 * q3 + q4 * q4);
    double w = q1 / n, x = q2 / n, y = q3 / n, z = q4 / n;
    o[ST_R0] = 1 - 2 * (y * y + z * z); o[ST_R1] = 2 * (x * y - w * z); o[ST_R2] = 2 * (x * z + w * y);
    o[ST_R3] = 2 * (x * y + w * z); o[ST_R4] = 1 - 2 * (x * x + z * z); o[ST_R5] = 2 * (y * z - w * x);
    o[ST_R6] = 2 * (x * z - w * y); o[ST_R7] = 2 * (y * z + w * x); o[ST_R8] = 1 - 2 * (x * x + y * y);
    o[ST_INVW] = exp(-p[11]);
    double smax = fmax(p[3], fmax(p[4], p[5]));
    o[ST_SUPP] = (-2.0 * log(kWEIGHT_CUTOFF)) * exp(2 * smax);
    o[ST_RHO] = sqrt(p[0] * p[0] + p[1] * p[1]);
    o[ST_KOFF] = d.kind == KS_KNOT21 ? double(d.koff + 4 * d.nk * i) : 0.0;
    o[ST_NK] = d.kind == KS_KNOT21 ? double(d.nk) : 0.0;
    if (d.kind == KS_KNOT21) {
        // every interpolated centre lies in the box of the knots: a point farther than the box's
        // half-diagonal plus the support radius from its centre is outside the support at any time
        const double* kn = d.knots + d.koff + 4 * d.nk * i;
        double lo[3], hi[3], half2 = 0.0;
        for (int q = 0; q < 3; ++q) {
            lo[q] = hi[q] = kn[(q + 1) * d.nk];
            for (int k = 1; k < d.nk; ++k) { lo[q] = fmin(lo[q], kn[(q + 1) * d.nk + k]); hi[q] = fmax(hi[q], kn[(q + 1) * d.nk + k]); }
            half2 += 0.25 * (hi[q] - lo[q]) * (hi[q] - lo[q]);
        }
        o[ST_CX] = 0.5 * (lo[0] + hi[0]); o[ST_CY] = 0.5 * (lo[1] + hi[1]); o[ST_CZ] = 0.5 * (lo[2] + hi[2]);
        const double rb = sqrt(half2) + sqrt(o[ST_SUPP]);
        o[ST_RHO] = rb * rb;   // the bounding radius squared (knot splats use no pattern circle)
    }
    if (d.kind == KS_THIN14) { o[ST_LOGA] = p[12]; return; }
    o[ST_NE] = exp(p[12]);
    double Bmag, thB, phB, u1, u2, u3;
    if (d.kind == KS_THERMAL21 || d.kind == KS_KNOT21) {
        double Te = exp(p[13]);
        o[ST_TE] = Te;
        double k0, k1;
        besselk01(1.0 / Te, k0, k1);
        double xb = 1.0 / Te;
        double k2 = k0 + 2.0 * k1 / xb;
        o[ST_F0] = k2 > 0 ? k0 / k2 : 1.0;
        o[ST_KR] = k2 > 0 ? k1 / k2 : 1.0;
        Bmag = exp(p[14]); thB = p[15]; phB = p[16]; u1 = p[17]; u2 = p[18]; u3 = p[19];
    } else {
        Bmag = exp(p[15]); thB = p[16]; phB = p[17]; u1 = p[18]; u2 = p[19]; u3 = p[20];
        if (d.kind == KS_POWERLAW22) {
            double pp = p[13], gmin = exp(p[14]);
            o[ST_P] = pp; o[ST_GMIN] = gmin; o[ST_GMAX] = d.gmax;
            o[ST_GSPAN] = pow(gmin, 1 - pp) - pow(d.gmax, 1 - pp);
            o[ST_GAMJ] = tgamma((3 * pp - 1) / 12) * tgamma((3 * pp + 19) / 12);
            o[ST_GAMA] = tgamma((3 * pp + 2) / 12) * tgamma((3 * pp + 22) / 12);
        } else {
            double kap = p[13], wk = exp(p[14]);
            o[ST_KAP] = kap; o[ST_W] = wk; o[ST_HYP] = d.hyp ? d.hyp[i] : 0.0;
            o[ST_G43] = tgamma(kap - 4.0 / 3); o[ST_G2] = tgamma(kap - 2);
            o[ST_GQ] = tgamma(kap / 4 - 1.0 / 3); o[ST_GP] = tgamma(kap / 4 + 4.0 / 3);
            o[ST_GK2] = tgamma(2 + kap / 2);
            double k0, k1;
            besselk01(1.0 / wk, k0, k1);
            double xb = 1.0 / wk;
            double k2 = k0 + 2.0 * k1 / xb;
            o[ST_KB] = k0 / (k2 + 1e-40);
        }
    }
    double B[3] = {Bmag * sin(thB) * cos(phB), Bmag * sin(thB) * sin(phB), Bmag * cos(thB)};
    double Bn = sqrt(B[0] * B[0] + B[1] * B[1] + B[2] * B[2]);
    o[ST_BMAG] = Bmag;
    if (Bn > 0) { o[ST_BHX] = B[0] / Bn; o[ST_BHY] = B[1] / Bn; o[ST_BHZ] = B[2] / Bn; o[ST_BZERO] = 0.0; }
    else { o[ST_BHX] = 0; o[ST_BHY] = 0; o[ST_BHZ] = 1; o[ST_BZERO] = 1.0; }
    o[ST_U1] = u1; o[ST_U2] = u2; o[ST_U3] = u3;
}

// ---- kernels: the fused march with its consumers -----------------------------------------------------

template <class T>
__device__ __forceinline__ void ks_coords(T a, T r, T th, T ph, T& x, T& y, T& z, T& sth, T& cth) {
    T temp = sqrt(T(1) - a * a);
    T rp = T(1) + temp, rm = T(1) - temp;
    T phks = ph + a / (T(2) * temp) * log(fabs((r - rp + keps<T>()) / (r - rm + keps<T>()))) - atan2(a, r);
    sth = sin(th); cth = cos(th);
    T sp = sin(phks), cp = cos(phks);
    x = r * sth * cp; y = r * sth * sp; z = r * cth;
}

}  // namespace

#include "ks_mixed.cuh"

namespace {

struct StoreSink {
    double *t, *r, *th, *ph; unsigned char* fl;
    long long npix, j;
    __device__ void operator()(int k, const Sample<double>& s) {
        long long q = (long long)(k - 1) * npix + j;
        t[q] = s.t; r[q] = s.r; th[q] = s.theta; ph[q] = s.phi;
        fl[q] = (s.ok ? 1 : 0) | (s.nur ? 2 : 0) | (s.nutheta ? 4 : 0);
    }
};

__global__ void k_march_store(PlanView P, Spacetime st, long long npix, double* t, double* r, double* th, double* ph,
                              unsigned char* fl, double* resid_t, double* resid_phi) {
    long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= npix) return;
    MarchRay<double> R = load_ray<double>(P, st, j);
    StoreSink sink{t, r, th, ph, fl, npix, j};
    double rt, rp;
    march(P, st, j, R, sink, rt, rp);
    resid_t[j] = rt; resid_phi[j] = rp;
}

// ThinRenderer (Splats.jl:113-128)
template <class T>
struct ThinSink {
    const T* tab; int nsplat; T t_obs; T a, rh_lo; T dtau; T acc;
    T eta, lam;
    __device__ void operator()(int, const Sample<T>& s) {
        if (!(s.ok && rh_lo < s.r && s.r < T(1e3))) return;
        T x, y, z, sth, cth;
        ks_coords(a, s.r, s.theta, s.phi, x, y, z, sth, cth);
        T t = t_obs - s.t;
        T jt = T(0);
        for (int i = 0; i < nsplat; ++i) {
            const T* p = tab + i * ST_COUNT;
            T q;
            splat_exponent(p, t, x, y, z, false, q);
            jt += exp(p[ST_LOGA] - q);
        }
        SampleFrame<T> F = sample_frame(a, s.r, s.theta, sth, cth, eta, lam, s.nur, s.nutheta);
        T g = T(1) / F.pz[0];
        T Sg = s.r * s.r + a * a * cth * cth;
        acc += g * g * jt * Sg * dtau;
    }
};

template <class T>
__global__ void k_thin(PlanView P, Spacetime st, long long npix, const double* __restrict__ tab64, int nsplat, double t_obs,
                       const long long* __restrict__ perm, double* __restrict__ out, double* __restrict__ resid_t,
                       double* __restrict__ resid_phi) {
    extern __shared__ __align__(16) unsigned char smem[];
    T* tab = reinterpret_cast<T*>(smem);
    for (int q = threadIdx.x; q < nsplat * ST_COUNT; q += blockDim.x) tab[q] = T(tab64[q]);
    __syncthreads();
    long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= npix) return;
    MarchRay<T> R = load_ray<T>(P, st, j);
    ThinSink<T> sink{tab, nsplat, T(t_obs), T(st.a), T(st.rh * (1 + 1e-3)), T(R.dtau), T(0), R.eta, R.lam};
    double rt, rp;
    march(P, st, j, R, sink, rt, rp);
    out[perm ? perm[j] : j] = double(sink.acc);   // sorted order, or screen order through the permutation
    if (resid_t) { resid_t[j] = rt; resid_phi[j] = rp; }
}

// The allocation-free thin-image variant (ks_thin_image_noalloc) keeps its splat table in this
// file-scope device array instead of a context buffer and runs k_thin with the image written straight
// into the caller's buffer. Every GPU that loads the library holds the array until the process exits;
// every call overwrites the first nsplat rows before reading them; calls that overlap on the GPU (two
// streams, two host threads) share it and race.
constexpr int kNoAllocMaxSplats = 256;
static __device__ __align__(256) double g_noalloc_tab[kNoAllocMaxSplats * ST_COUNT];

// RadiativeTransport over a concatenated splat table (transport.jl:171-198, polarized.jl:121-150,
// populations.jl:70-104), CH (t_obs, nu) combinations per thread sharing the march.
template <class T, int CH>
struct PolSink {
    const T* tab; int ntot;
    const T* knots;   // the knot array of knot splats (after the table)
    T t_obs[CH], nu[CH], nuh[CH], Lnu[CH];
    int nc;
    T a, rh_lo, dtau, alpha, beta, eta, lam, a_sin_tho, slab;
    int nmax;
    T P[CH][16], S[CH][4];
    T zprev; int wn; bool inside, crossed, zset;
    // event counts of this thread (the algorithmic-work model of the roofline): samples, valid
    // samples, splat tests, weights evaluated, coefficient evaluations, frames, steps
    unsigned int ev[7];

    __device__ void init() {
        for (int q = 0; q < 7; ++q) ev[q] = 0;
        for (int c = 0; c < CH; ++c) {
            for (int q = 0; q < 16; ++q) P[c][q] = (q % 5 == 0) ? T(1) : T(0);
            for (int q = 0; q < 4; ++q) S[c][q] = T(0);
        }
        wn = 0; inside = false; crossed = false; zset = false; zprev = T(0);
    }

    __device__ void wind(T z) {   // step.jl:379-398
        if (!zset) { zprev = z; zset = true; inside = fabs(z) < slab; crossed = false; return; }
        bool inside_now = fabs(z) < slab;
        bool crossing = zprev * z < T(0);
        if (inside || inside_now) {
            crossed = crossed || crossing;
            if (inside && !inside_now) { if (crossed) wn += 1; crossed = false; }
            else if (!inside && inside_now) { crossed = crossing; }
            inside = inside_now;
        } else if (crossing) {
            wn += 1;
        }
        zprev = z;
    }

    __device__ void operator()(int, const Sample<T>& s) {
        ev[0]++;
        if (!(s.ok && s.r > rh_lo)) return;
        ev[1]++;
        if (nmax >= 0) {
            wind(s.r * cos(s.theta));
            if (wn > nmax) return;
        }
        T x, y, z, sth, cth;
        ks_coords(a, s.r, s.theta, s.phi, x, y, z, sth, cth);
        T j4[CH][4], a4[CH][4], r3[CH][3];
        bool active[CH];
        for (int c = 0; c < CH; ++c) {
            active[c] = false;
            for (int q = 0; q < 4; ++q) { j4[c][q] = T(0); a4[c][q] = T(0); }
            for (int q = 0; q < 3; ++q) r3[c][q] = T(0);
        }
        bool have_frame = false;
        SampleFrame<T> F;
        for (int i = 0; i < ntot; ++i) {
            const T* p = tab + i * ST_COUNT;
            const int kind = int(p[ST_KIND]);
            bool fr_done = false;
            LFrame<T> lf;
            for (int c = 0; c < CH; ++c) {
                if (c >= nc) break;
                T t = t_obs[c] - s.t;
                T q;
                ev[2]++;
                if (!any_exponent(p, knots, t, x, y, z, q)) continue;
                ev[3]++;
                T G = exp(-q);
                if (!(G > T(kWEIGHT_CUTOFF))) continue;
                if (!have_frame) { F = sample_frame(a, s.r, s.theta, sth, cth, eta, lam, s.nur, s.nutheta); have_frame = true; }
                ev[4]++;
                if (!fr_done) {
                    ev[5]++;
                    lf = local_frame(F, p[ST_U1], p[ST_U2], p[ST_U3], p[ST_BHX], p[ST_BHY], p[ST_BHZ], p[ST_BZERO] != T(0),
                                     alpha, beta, a_sin_tho);
                    fr_done = true;
                }
                T nuf = nu[c] / lf.g;
                T thb = acos(fmin(T(1), fmax(T(-1), lf.cosB)));
                T ne = p[ST_NE] * G;
                Coef<T> cf;
                if (kind == KS_POWERLAW22)
                    cf = powerlaw(ne, p[ST_P], p[ST_GMIN], p[ST_GSPAN], p[ST_GAMJ], p[ST_GAMA], p[ST_BMAG], nuf, thb);
                else if (kind == KS_KAPPA22)
                    cf = kappa(ne, p[ST_KAP], p[ST_W], p[ST_HYP], p[ST_G43], p[ST_G2], p[ST_GQ], p[ST_GP], p[ST_GK2], p[ST_KB], p[ST_BMAG], nuf, thb);
                else
                    cf = thermal(ne, p[ST_TE], p[ST_F0], p[ST_KR], p[ST_BMAG], nuf, thb);
                // screen_coefficients (transport.jl:265-270): cap, invariants at nu/g, rotate by 2 chi
                if (!(cf.jI > T(0) || cf.aI > T(0) || cf.rQ != T(0) || cf.rV != T(0))) continue;
                T fe = cap_factor(cf.jI, cf.jQ, cf.jV, T(0.99));
                T fa = cap_factor(cf.aI, cf.aQ, cf.aV, T(0.99));
                T nh = nuf / T(kNU0);
                T i2 = T(1) / (nh * nh);
                T s2c = lf.s2c, c2c = lf.c2c;
                T jQ = cf.jQ * fe * i2, aQ = cf.aQ * fa * nh, rQ = cf.rQ * nh;
                j4[c][0] += cf.jI * i2; j4[c][1] += jQ * c2c; j4[c][2] += jQ * s2c; j4[c][3] += cf.jV * fe * i2;
                a4[c][0] += nh * cf.aI; a4[c][1] += aQ * c2c; a4[c][2] += aQ * s2c; a4[c][3] += cf.aV * fa * nh;
                r3[c][0] += rQ * c2c; r3[c][1] += rQ * s2c; r3[c][2] += nh * cf.rV;
                active[c] = true;
            }
        }
        T Sg = s.r * s.r + a * a * cos(s.theta) * cos(s.theta);
        for (int c = 0; c < CH; ++c) {
            if (c >= nc || !active[c]) continue;
            T Dl = Lnu[c] * Sg * dtau;
            ev[6]++;
            T O[16], E[4];
            transfer_step(c_moments, j4[c], a4[c], r3[c], Dl, O, E);
            // advance (step.jl:347): S += P E, P = P O
            T Pn[16];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                S[c][r] += P[c][4 * r] * E[0] + P[c][4 * r + 1] * E[1] + P[c][4 * r + 2] * E[2] + P[c][4 * r + 3] * E[3];
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    Pn[4 * r + q] = P[c][4 * r] * O[q] + P[c][4 * r + 1] * O[4 + q] + P[c][4 * r + 2] * O[8 + q] + P[c][4 * r + 3] * O[12 + q];
            }
#pragma unroll
            for (int q = 0; q < 16; ++q) P[c][q] = Pn[q];
        }
    }
};

template <class T, int CH>
__global__ void __launch_bounds__(kBlock) k_polarized(PlanView P, Spacetime st, long long npix, const double* __restrict__ tab64, int ntot,
                                                      const double* __restrict__ ct, const double* __restrict__ cnu, int ncombo, double L,
                                                      int nmax, double slab, double* __restrict__ out, double* __restrict__ resid_t,
                                                      double* __restrict__ resid_phi, unsigned long long* __restrict__ counters, int nkv) {
    extern __shared__ __align__(16) unsigned char smem[];
    T* tab = reinterpret_cast<T*>(smem);
    for (int q = threadIdx.x; q < ntot * ST_COUNT + nkv; q += blockDim.x) tab[q] = T(tab64[q]);
    __syncthreads();
    long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= npix) return;
    const int c0 = blockIdx.y * CH;
    MarchRay<T> R = load_ray<T>(P, st, j);
    PolSink<T, CH> sink;
    sink.tab = tab; sink.ntot = ntot; sink.knots = tab + ntot * ST_COUNT;
    sink.nc = min(CH, ncombo - c0);
    for (int c = 0; c < CH; ++c) {
        int cc = min(c0 + c, ncombo - 1);
        sink.t_obs[c] = T(ct[cc]); sink.nu[c] = T(cnu[cc]);
        double nh = cnu[cc] / kNU0;
        sink.nuh[c] = T(nh);
        sink.Lnu[c] = T(L / nh);
    }
    sink.a = T(st.a); sink.rh_lo = T(st.rh * (1 + 1e-3)); sink.dtau = T(R.dtau);
    sink.alpha = T(P.get(PF_ALPHA, j)); sink.beta = T(P.get(PF_BETA, j)); sink.eta = R.eta; sink.lam = R.lam;
    sink.a_sin_tho = T(st.a * sin(st.thetao)); sink.slab = T(slab); sink.nmax = nmax;
    sink.init();
    double rt, rp;
    march(P, st, j, R, sink, rt, rp);
    for (int c = 0; c < CH; ++c) {
        if (c >= sink.nc) break;
        double n3 = double(sink.nuh[c]) * double(sink.nuh[c]) * double(sink.nuh[c]);
        double* o = out + ((long long)(c0 + c) * npix + j) * 4;
        o[0] = double(sink.S[c][0]) * n3; o[1] = double(sink.S[c][1]) * n3;
        o[2] = double(sink.S[c][2]) * n3; o[3] = double(sink.S[c][3]) * n3;
    }
    if (blockIdx.y == 0 && resid_t) { resid_t[j] = rt; resid_phi[j] = rp; }
    if (counters) {
        // samples are counted once per (ray, combo) as the metric counts them
        atomicAdd(&counters[0], (unsigned long long)sink.ev[0] * sink.nc);
        for (int q = 1; q < 7; ++q) atomicAdd(&counters[q], (unsigned long long)sink.ev[q]);
    }
}

// ---- ipole's RIAF as a fluid model of the polarized consumer ------------------------------------
// The reference's test/riaf_model.jl: a thick disk with power-law density and temperature, a
// toroidal field of equipartition-like strength, Keplerian rotation outside the ISCO and the plunge
// with the ISCO's conserved energy and angular momentum inside it, thermal synchrotron (Pandya
// emissivities when `pandya`, ipole's emission_type 1). One element, evaluated at every sample.
struct RiafModel { double nth0, Te0, disk_h, pow_nth, pow_T, Ne_unit, Te_unit, eps, r_isco, rout; int pandya; };

constexpr double kMP = 1.67262171e-24, kKBOL = 1.3806505e-16;   // constants.jl:3-12

// The coefficients and the local frame of the RIAF at the BL point (r, theta) of a sample, for the
// photon of the sample's frame F; false where the model is empty (r <= r_h + 0.1 or r >= rout).
template <class T>
__device__ __forceinline__ bool riaf_element(const RiafModel& m, T a, T r, T th, T sth, T cth, const SampleFrame<T>& F, T alpha, T beta,
                                             T a_sin_tho, T nu, Coef<T>& cf, LFrame<T>& lf) {
    const T rh = T(1) + sqrt(T(1) - a * a);
    if (!(r > rh + T(0.1) && r < T(m.rout))) return false;
    // density, temperature, field strength (ipole's get_model_ne / thetae / b)
    const T zc = r * cth, rc = r * sth;
    const T hh = T(m.disk_h);
    const T n = T(m.nth0) * exp(-zc * zc / T(2) / rc / rc / hh / hh) * pow(r, T(m.pow_nth)) * T(m.Ne_unit);
    const T Te = T(m.Te0) * pow(r, T(m.pow_T)) * T(m.Te_unit) * T(kKBOL) / (T(kME) * T(kCL) * T(kCL));
    T bmag = sqrt(T(8) * kpi<T>() * T(m.eps) * n * T(kMP) * T(kCL) * T(kCL) / T(6) / r);
    if (bmag == T(0)) bmag = T(1e-6);
    // the Boyer-Lindquist metric at (r, theta) and at (r_isco, theta)
    const T s2 = sth * sth;
    auto gdd = [&](T rr, T& gtt, T& gtp, T& grr, T& gpp) {
        const T S = rr * rr + a * a * cth * cth, D = rr * rr - T(2) * rr + a * a;
        gtt = -(T(1) - T(2) * rr / S); gtp = -T(2) * a * rr * s2 / S; grr = S / D;
        gpp = (rr * rr + a * a + T(2) * a * a * rr * s2 / S) * s2;
    };
    T gtt, gtp, grr, gpp;
    gdd(r, gtt, gtp, grr, gpp);
    T om, ur;
    const T risco = T(m.r_isco);
    if (r < risco) {
        // the plunge: the ISCO's conserved e, l (ipole get_model_fourv)
        T itt, itp, irr, ipp;
        gdd(risco, itt, itp, irr, ipp);
        const T wis = T(1) / (pow(risco, T(1.5)) + a);
        const T nrm = sqrt(-(itt + T(2) * wis * itp + wis * wis * ipp));
        const T u0 = T(1) / nrm, u3 = wis / nrm;
        const T e = itt * u0 + itp * u3, l = itp * u0 + ipp * u3;
        // the inverse metric at (r, theta)
        const T S = r * r + a * a * cth * cth, D = r * r - T(2) * r + a * a;
        const T A = (r * r + a * a) * (r * r + a * a) - a * a * D * s2;
        const T utt = -A / (S * D), utp = -T(2) * a * r / (S * D), urr = D / S, upp = (D - a * a * s2) / (S * D * s2);
        const T Kcon = utt * e * e + T(2) * utp * e * l + upp * l * l;
        const T q = -(T(1) + Kcon) / urr;
        const T urk = -(q > T(0) ? sqrt(q) : T(0));
        const T c0 = utt * e + utp * l, c3 = utp * e + upp * l;
        om = c3 / c0;
        ur = urr * urk;
    } else {
        om = T(1) / (pow(r, T(1.5)) + a);
        ur = T(0);
    }
    const T K = gtt + T(2) * om * gtp + om * om * gpp;
    const T q2 = -(T(1) + ur * ur * grr) / K;
    const T ut = q2 > T(0) ? sqrt(q2) : T(0);
    const T u[4] = {ut, ur, T(0), om * ut};
    // toroidal field projected orthogonal to u, normalised to bmag
    const T BdotU = gtp * u[0] + gpp * u[3];
    T b[4] = {BdotU * u[0], BdotU * u[1], T(0), T(1) + BdotU * u[3]};
    const T bb = gtt * b[0] * b[0] + T(2) * gtp * b[0] * b[3] + grr * b[1] * b[1] + gpp * b[3] * b[3];
    const T bs = bmag / sqrt(bb);
#pragma unroll
    for (int k = 0; k < 4; ++k) b[k] *= bs;
    // ZAMO components (t, r, phi, -theta): lapse, sqrt(S/D), varpi (. - omega_frame t), -sqrt(S)
    const T S = r * r + a * a * cth * cth, D = r * r - T(2) * r + a * a;
    const T A = (r * r + a * a) * (r * r + a * a) - a * a * D * s2;
    const T lapse = sqrt(S * D / A), omf = T(2) * a * r / A, varpi = sqrt(A / S) * sth, sSD = sqrt(S / D);
    const T u1 = sSD * u[1], u2 = varpi * (u[3] - omf * u[0]), u3 = T(0);
    const T bz0 = lapse * b[0], bz1 = sSD * b[1], bz2 = varpi * (b[3] - omf * b[0]), bz3 = T(0);
    // the field in the fluid frame: boost_zamo_to_fluid(u) (frames.jl:31-41)
    const T gam = sqrt(T(1) + u1 * u1 + u2 * u2 + u3 * u3), qf = T(1) / (gam + T(1));
    const T ub = u1 * bz1 + u2 * bz2 + u3 * bz3;
    const T f1 = -u1 * bz0 + bz1 + u1 * ub * qf, f2 = -u2 * bz0 + bz2 + u2 * ub * qf, f3 = -u3 * bz0 + bz3 + u3 * ub * qf;
    const T fn = sqrt(f1 * f1 + f2 * f2 + f3 * f3);
    const bool bzero = !(fn > T(0));
    lf = local_frame(F, u1, u2, u3, bzero ? T(0) : f1 / fn, bzero ? T(0) : f2 / fn, bzero ? T(1) : f3 / fn, bzero, alpha, beta, a_sin_tho);
    const T nuf = nu / lf.g;
    T sb, cb;
    if constexpr (is_f32<T>) {
        pitch_sc(lf.cosB, sb, cb);
    } else {
        const T thb = acos(fmin(T(1), fmax(T(-1), lf.cosB)));
        sb = sin(thb); cb = cos(thb);
    }
    // Bessel ratios at 1/Theta_e (K2 = K0 + 2 K1 / x), FP64
    double k0, k1;
    const double xb = 1.0 / double(Te);
    besselk01(xb, k0, k1);
    const double k2 = k0 + 2.0 * k1 / xb;
    const T f0 = k2 > 0 ? T(k0 / k2) : T(1), kr = k2 > 0 ? T(k1 / k2) : T(1);
    cf = thermal_cs(n, Te, f0, kr, bmag, nuf, sb, cb);
    if (m.pandya && sb > T(0)) {
        T jI, jQ, jV;
        pandya_emissivities(n, Te, bmag, nuf, sb, cb, jI, jQ, jV);
        const T Bn = planck(nuf, Te);
        const T invB = Bn > T(0) ? T(1) / Bn : T(0);
        cf.jI = jI; cf.jQ = jQ; cf.jV = jV; cf.aI = jI * invB; cf.aQ = jQ * invB; cf.aV = jV * invB;
    }
    return true;
}

// RadiativeTransport of the RIAF at one frequency (stokes_image, test/test_polarized.jl:54-61): the
// FP64 march, the element and the step in T.
template <class T>
struct RiafSink {
    RiafModel m;
    T nu, Lnu;
    T a, rh_lo, dtau, alpha, beta, eta, lam, a_sin_tho;
    T P[16], S[4];
    unsigned int ev[7];

    __device__ void init() {
        for (int q = 0; q < 16; ++q) P[q] = (q % 5 == 0) ? T(1) : T(0);
        for (int q = 0; q < 4; ++q) S[q] = T(0);
        for (int q = 0; q < 7; ++q) ev[q] = 0;
    }

    __device__ void operator()(int, const Sample<double>& s) {
        ev[0]++;
        if (!(s.ok && T(s.r) > rh_lo)) return;
        ev[1]++;
        const T r = T(s.r), th = T(s.theta);
        const T sth = sin(th), cth = cos(th);
        const SampleFrame<T> F = sample_frame(a, r, th, sth, cth, eta, lam, s.nur, s.nutheta);
        Coef<T> cf;
        LFrame<T> lf;
        ev[2]++;
        if (!riaf_element(m, a, r, th, sth, cth, F, alpha, beta, a_sin_tho, nu, cf, lf)) return;
        ev[3]++; ev[4]++; ev[5]++;
        // screen_coefficients (transport.jl:265-270): cap, invariants at nu/g, rotate by 2 chi
        if (!(cf.jI > T(0) || cf.aI > T(0) || cf.rQ != T(0) || cf.rV != T(0))) return;
        const T fe = cap_factor(cf.jI, cf.jQ, cf.jV, T(0.99));
        const T fa = cap_factor(cf.aI, cf.aQ, cf.aV, T(0.99));
        const T nh = nu / lf.g / T(kNU0);
        const T i2 = T(1) / (nh * nh);
        const T jQ = cf.jQ * fe * i2, aQ = cf.aQ * fa * nh, rQ = cf.rQ * nh;
        const T j4[4] = {cf.jI * i2, jQ * lf.c2c, jQ * lf.s2c, cf.jV * fe * i2};
        const T a4[4] = {nh * cf.aI, aQ * lf.c2c, aQ * lf.s2c, cf.aV * fa * nh};
        const T r3[3] = {rQ * lf.c2c, rQ * lf.s2c, nh * cf.rV};
        const T Dl = Lnu * (r * r + a * a * cth * cth) * dtau;
        ev[6]++;
        T O[16], E[4];
        transfer_step(c_moments, j4, a4, r3, Dl, O, E);
        T Pn[16];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            S[i] += P[4 * i] * E[0] + P[4 * i + 1] * E[1] + P[4 * i + 2] * E[2] + P[4 * i + 3] * E[3];
#pragma unroll
            for (int q = 0; q < 4; ++q)
                Pn[4 * i + q] = P[4 * i] * O[q] + P[4 * i + 1] * O[4 + q] + P[4 * i + 2] * O[8 + q] + P[4 * i + 3] * O[12 + q];
        }
#pragma unroll
        for (int q = 0; q < 16; ++q) P[q] = Pn[q];
    }
};

// One thread per ray, one frequency per grid row: out[(f npix + j) 4 + stokes] in sorted order.
template <class T>
__global__ void __launch_bounds__(kBlock) k_riaf(PlanView P, Spacetime st, long long npix, RiafModel m, const double* __restrict__ nus,
                                                 double L, double* __restrict__ out, unsigned long long* __restrict__ counters) {
    const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= npix) return;
    const int f = blockIdx.y;
    MarchRay<double> R = load_ray<double>(P, st, j);
    RiafSink<T> sink;
    sink.m = m;
    const double nh = nus[f] / kNU0;
    sink.nu = T(nus[f]); sink.Lnu = T(L / nh);
    sink.a = T(st.a); sink.rh_lo = T(st.rh * (1 + 1e-3)); sink.dtau = T(R.dtau);
    sink.alpha = T(P.get(PF_ALPHA, j)); sink.beta = T(P.get(PF_BETA, j)); sink.eta = T(R.eta); sink.lam = T(R.lam);
    sink.a_sin_tho = T(st.a * sin(st.thetao));
    sink.init();
    double rt, rp;
    march(P, st, j, R, sink, rt, rp);
    double* o = out + ((long long)f * npix + j) * 4;
    const double n3 = nh * nh * nh;
    o[0] = double(sink.S[0]) * n3; o[1] = double(sink.S[1]) * n3; o[2] = double(sink.S[2]) * n3; o[3] = double(sink.S[3]) * n3;
    if (counters) {
        atomicAdd(&counters[0], (unsigned long long)sink.ev[0]);
        for (int q = 1; q < 7; ++q) atomicAdd(&counters[q], (unsigned long long)sink.ev[q]);
    }
}

}  // namespace

#include "ks_adjoint.cuh"
#include "ks_spacetime.cuh"

namespace {

__global__ void k_inverse_perm(const long long* __restrict__ perm, long long npix, long long* __restrict__ inv) {
    long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j < npix) inv[perm[j]] = j;
}

// sorted slot -> output order, for `nvec` blocks of npix rows of `width` doubles
__global__ void k_unsort(const double* __restrict__ src, const long long* __restrict__ perm, long long npix, int width, int nvec,
                         int to_screen, double* __restrict__ dst) {
    long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    long long total = npix * nvec;
    if (q >= total) return;
    long long v = q / npix, j = q % npix;
    long long dj = to_screen ? perm[j] : j;
    for (int w = 0; w < width; ++w) dst[(v * npix + dj) * width + w] = src[(v * npix + j) * width + w];
}

}  // namespace

// ---- the context ----------------------------------------------------------------------------------------

struct DevBuf {
    void* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;   // one owner per allocation
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    cudaError_t ensure(size_t bytes) {
        if (bytes <= n) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr; n = 0;
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e == cudaSuccess) n = bytes;
        return e;
    }
    void release() { if (p) cudaFree(p); p = nullptr; n = 0; }
    template <class U> U* as() const { return reinterpret_cast<U*>(p); }
};

struct ks_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    long long npix = 0, npad = 0;
    int nalpha = 0, nbeta = 0;
    bool regenerated = false;
    Spacetime st{};
    DevBuf alpha, beta, key, key2, idx, perm, plan, nanch, aoff, anchors, resid_t, resid_phi, scratch;
    DevBuf tab, combos, out_sorted, stage_in, stage_out, counters, seg_out, work, stream_buf;
    DevBuf inv_perm, dft_tu, dft_tv, dft_a, dft_t, dft_c, dft_s, dft_in[8], dft_partial;
    // adjoint: gradient table, stored FP64 samples (plain path), cutoffs, tails, per-ray slots,
    // seeds, chi^2 partials; mixed path: per-sample states, activity, segment bounds, unit partials
    DevBuf gtab, samples, kstop, tails, slots, dgrad, seeds, chi_part, chi_val, dstage;
    DevBuf adj_state, adj_act, adj_bnd, adj_unit, adj_part, jvp_tab, jvp_in, jvp_out, st_buf;
    DevBuf tab32;     // the splat table and knot array in FP32, padded to 16 bytes (the TMA staging source)
    DevBuf errflag;   // set by a kernel whose bounded wait gave up
    cudaGraph_t graph = nullptr;          // ks_render_graph_capture: one mixed render of device-resident sets
    cudaGraphExec_t graph_exec = nullptr;
    cudaGraph_t cgraph = nullptr;         // ks_chi2_gradient_graph_capture: one mixed chi^2 + gradient evaluation
    cudaGraphExec_t cgraph_exec = nullptr;
    std::vector<void*> cgraph_bufs;
    bool capturing = false;               // inside that capture: no timing events
    int stage_test = 0;                   // ks_set_stage_test
    std::vector<void*> graph_bufs;        // the buffers the graph uses, as captured (a replay checks them)
    bool samples_ready = false;
    int tune_nt = 0, tune_units = 0;        // the autotuner's choice for the mixed forward (0: the default)
    int nkv = 0;                            // knot values after the splat table in `tab`
    MixedJob last_job{};                    // the segmentation of the last mixed forward pass
    float* fwd_gstate = nullptr;            // set during the adjoint's forward pass only
    unsigned char* fwd_gact = nullptr;
    double adjoint_ms = 0.0;
    long long adjoint_launches = 0;
    bool count_events = false;
    int tensor_path = 0;  // 3xTF32 GEMMs: 0 tcgen05 (k_gemm_tc), 1 mma.sync (k_gemm_3xtf32); ks_set_tensor_path
    bool geo64 = false;   // mixed path: the FP64 march feeds the FP32 transport (KS_MIXED_GEO64) instead of the FP32 march
    long long total_anchors = 0;
    int max_nanch = 0;
    long long ranges[6] = {0, 0, 0, 0, 0, 0};
    // timing of the render kernels (CUDA events on the context stream)
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t evc0 = nullptr, evc1 = nullptr;   // around k_consume (the mixed path's dominant kernel)
    cudaEvent_t evg0 = nullptr, evg1 = nullptr;   // around each 3xTF32 GEMM (outside graph captures)
    double gemm_ms = 0.0, gemm_flops = 0.0;       // ks_gemm_stats: device time and tensor-core flops (3 x 2 M N K)
    long long gemm_launches = 0;
    bool consume_timed = false;
    double consume_ms = 0.0;
    long long consume_launches = 0;
    double kernel_ms = 0.0;
    long long kernel_launches = 0;
    long long launches = 0;
};

namespace {

int fail(ks_context* c, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return code;
}

int cuda_fail(ks_context* c, cudaError_t e, const char* what) {
    if (e == cudaErrorMemoryAllocation) return fail(c, KS_ERR_OUT_OF_MEMORY, "%s: %s", what, cudaGetErrorString(e));
    return fail(c, KS_ERR_DEVICE, "%s: %s", what, cudaGetErrorString(e));
}

#define KS_CUDA(ctx, call)                                            \
    do {                                                              \
        cudaError_t e_ = (call);                                      \
        if (e_ != cudaSuccess) return cuda_fail((ctx), e_, #call);    \
    } while (0)

bool is_device_ptr(const void* p) {
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) { cudaGetLastError(); return false; }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Make `src` (host or device, `bytes`) available on the device: returns the device pointer.
int stage_in(ks_context* c, DevBuf& buf, const void* src, size_t bytes, const void** dev) {
    if (is_device_ptr(src)) { *dev = src; return KS_OK; }
    KS_CUDA(c, buf.ensure(bytes));
    KS_CUDA(c, cudaMemcpyAsync(buf.p, src, bytes, cudaMemcpyHostToDevice, c->stream));
    *dev = buf.p;
    return KS_OK;
}

void init_constants() {
    MomentCoeffs mc;
    for (int n = 0; n < 10; ++n) {
        double fact = 1.0;
        for (int m = 0; m < 24; ++m) {
            if (m > 0) fact *= m;
            mc.c[n][m] = ((m % 2) ? -1.0 : 1.0) / (fact * (n + m + 1));
            mc.cf[n][m] = float(mc.c[n][m]);
        }
    }
    cudaMemcpyToSymbol(c_moments, &mc, sizeof mc);
    // 16-point Gauss-Legendre nodes on [-1, 1] (Newton on P_16)
    double x[16], w[16];
    const int n = 16;
    for (int i = 0; i < n; ++i) {
        double z = std::cos(kPi * (i + 0.75) / (n + 0.5)), dp = 0.0;
        for (int it = 0; it < 100; ++it) {
            double p1 = 1.0, p2 = 0.0;
            for (int jj = 1; jj <= n; ++jj) { double p3 = p2; p2 = p1; p1 = ((2.0 * jj - 1.0) * z * p2 - (jj - 1.0) * p3) / jj; }
            dp = n * (z * p1 - p2) / (z * z - 1.0);
            double dz = p1 / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-17) break;
        }
        double p1 = 1.0, p2 = 0.0;
        for (int jj = 1; jj <= n; ++jj) { double p3 = p2; p2 = p1; p1 = ((2.0 * jj - 1.0) * z * p2 - (jj - 1.0) * p3) / jj; }
        dp = n * (z * p1 - p2) / (z * z - 1.0);
        x[i] = z; w[i] = 2.0 / ((1.0 - z * z) * dp * dp);
    }
    cudaMemcpyToSymbol(c_gl_x, x, sizeof x);
    cudaMemcpyToSymbol(c_gl_w, w, sizeof w);
}

unsigned nblocks(long long n, int b = kBlock) { return unsigned((n + b - 1) / b); }

PlanView plan_view(ks_context* c) {
    PlanView P;
    P.f = c->plan.as<double>(); P.npad = c->npad; P.anchors = c->anchors.as<double>(); P.anchor_off = c->aoff.as<long long>();
    return P;
}

int nrows_of(int kind) {
    switch (kind) {
        case KS_THIN14: return 14;
        case KS_THERMAL21: case KS_KNOT21: return 21;
        case KS_POWERLAW22: case KS_KAPPA22: return 22;
        default: return -1;
    }
}

// The concatenated splat table of a scene (and, with `grad`, the gradient table of its THERMAL21
// splats): validates the sets, stages each set's parameters and runs k_splat_table / k_grad_table.
int build_tables(ks_context* c, const ks_splat_set* sets, int nsets, int* ntot_out, bool grad) {
    int ntot = 0;
    for (int s = 0; s < nsets; ++s) {
        int nr = nrows_of(sets[s].kind);
        if (nr < 0 || sets[s].kind == KS_THIN14) return fail(c, KS_ERR_ARGUMENT, "set %d: unsupported kind %d", s, sets[s].kind);
        if (grad && sets[s].kind != KS_THERMAL21)
            return fail(c, KS_ERR_ARGUMENT, "set %d: the adjoint covers thermal polarized splats (KS_THERMAL21) only", s);
        if (sets[s].nsplat < 0 || (sets[s].nsplat > 0 && !sets[s].params)) return fail(c, KS_ERR_ARGUMENT, "set %d: bad parameters", s);
        if (sets[s].kind == KS_KAPPA22 && sets[s].nsplat > 0 && !sets[s].hyp) return fail(c, KS_ERR_ARGUMENT, "set %d: kappa sets need hyp", s);
        ntot += sets[s].nsplat;
    }
    // the knot array of the knot sets (trajectories.jl:80-111): per splat its times, x, y, z
    std::vector<double> kv;
    std::vector<int> koff(nsets, 0);
    for (int s = 0; s < nsets; ++s) {
        const ks_splat_set& S = sets[s];
        if (S.kind != KS_KNOT21 || S.nsplat == 0) continue;
        if (!S.knots || !S.knot_times || S.nknots < 1) return fail(c, KS_ERR_ARGUMENT, "set %d: knot splats need knots and knot times", s);
        const int nk = S.nknots;
        std::vector<double> ht(nk), hk(size_t(3) * nk * S.nsplat);
        KS_CUDA(c, cudaMemcpy(ht.data(), S.knot_times, ht.size() * sizeof(double), cudaMemcpyDefault));
        KS_CUDA(c, cudaMemcpy(hk.data(), S.knots, hk.size() * sizeof(double), cudaMemcpyDefault));
        for (int k = 0; k < nk; ++k)
            if (!std::isfinite(ht[k]) || (k > 0 && !(ht[k] > ht[k - 1]))) return fail(c, KS_ERR_ARGUMENT, "set %d: knot times must increase", s);
        for (double v : hk) if (!std::isfinite(v)) return fail(c, KS_ERR_NONFINITE, "set %d: non-finite knot", s);
        koff[s] = int(kv.size());
        for (int i = 0; i < S.nsplat; ++i) {
            kv.insert(kv.end(), ht.begin(), ht.end());
            for (int d = 0; d < 3; ++d)
                for (int k = 0; k < nk; ++k) kv.push_back(hk[d + 3 * (k + size_t(nk) * i)]);
        }
    }
    c->nkv = int(kv.size());
    KS_CUDA(c, c->tab.ensure((size_t(std::max(ntot, 1)) * ST_COUNT + kv.size()) * sizeof(double)));
    if (!kv.empty())
        KS_CUDA(c, cudaMemcpyAsync(c->tab.as<double>() + size_t(ntot) * ST_COUNT, kv.data(), kv.size() * sizeof(double),
                                   cudaMemcpyHostToDevice, c->stream));
    if (grad) KS_CUDA(c, c->gtab.ensure(size_t(std::max(ntot, 1)) * GT_COUNT * sizeof(double)));
    int first = 0;
    for (int s = 0; s < nsets; ++s) {
        const ks_splat_set& S = sets[s];
        if (S.nsplat == 0) continue;
        const int nr = nrows_of(S.kind);
        const void* dh = nullptr;
        // each set is staged into its own device buffer
        std::vector<double> hp(size_t(nr) * S.nsplat);
        KS_CUDA(c, cudaMemcpy(hp.data(), S.params, hp.size() * sizeof(double), cudaMemcpyDefault));
        for (double v : hp) if (!std::isfinite(v)) return fail(c, KS_ERR_NONFINITE, "set %d: non-finite parameter", s);
        DevBuf tmp;
        KS_CUDA(c, tmp.ensure(hp.size() * sizeof(double) + size_t(S.nsplat) * sizeof(double)));
        KS_CUDA(c, cudaMemcpyAsync(tmp.p, hp.data(), hp.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        if (S.kind == KS_KAPPA22) {
            double* hd = tmp.as<double>() + hp.size();
            KS_CUDA(c, cudaMemcpyAsync(hd, S.hyp, S.nsplat * sizeof(double), cudaMemcpyDefault, c->stream));
            dh = hd;
        }
        SetDesc d{S.kind, nr, S.nsplat, first, tmp.as<const double>(), (const double*)dh, S.gamma_max > 0 ? S.gamma_max : 1e5, koff[s],
                  S.kind == KS_KNOT21 ? S.nknots : 0, c->tab.as<const double>() + size_t(ntot) * ST_COUNT};
        k_splat_table<<<nblocks(S.nsplat, 64), 64, 0, c->stream>>>(d, c->tab.as<double>());
        c->launches++;
        KS_CUDA(c, cudaGetLastError());
        if (grad) {
            k_grad_table<<<nblocks(S.nsplat, 64), 64, 0, c->stream>>>(S.nsplat, first, tmp.as<const double>(), c->gtab.as<double>());
            c->launches++;
            KS_CUDA(c, cudaGetLastError());
        }
        KS_CUDA(c, cudaStreamSynchronize(c->stream));
        tmp.release();
        first += S.nsplat;
    }
    // the FP32 copy the mixed kernels stage into shared memory (a multiple of 16 bytes)
    {
        const long long nv = (long long)ntot * ST_COUNT + c->nkv;
        const long long np4 = std::max<long long>(4, (nv + 3) / 4 * 4);
        KS_CUDA(c, c->tab32.ensure(size_t(np4) * sizeof(float)));
        k_tab_f32<<<nblocks(np4, 256), 256, 0, c->stream>>>(nv, np4, c->tab.as<double>(), c->tab32.as<float>());
        c->launches++;
        KS_CUDA(c, cudaGetLastError());
    }
    *ntot_out = ntot;
    return KS_OK;
}

// A kernel's bounded wait that gave up (the device flag, cleared): KS_ERR_TIMEOUT. Bit 1: a mixed
// kernel's table-staging copy; bit 2: a wait of the tcgen05 GEMM.
int check_device_flag(ks_context* c, const char* what) {
    unsigned f = 0;
    KS_CUDA(c, cudaMemcpy(&f, c->errflag.p, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (f) {
        KS_CUDA(c, cudaMemset(c->errflag.p, 0, sizeof(unsigned)));
        return fail(c, KS_ERR_TIMEOUT, "%s: %s", what,
                    (f & 2u) ? "a wait of the tensor-core GEMM gave up" : "a shared-memory staging copy did not complete");
    }
    return KS_OK;
}

// The FP32 sample stream of every ray (k_stream: the FP32 march, or the FP64 march under
// KS_MIXED_GEO64), [k][field][npad]. Each ray is marched as up to eight segments, each starting
// at an anchor (a multiple of M samples). At 256 x 256, N = 1024 that is 6.9 waves of 16 warps per
// SM instead of 3.5 with four segments (the render 22.04 against 22.34 ms).
int launch_stream(ks_context* c) {
    const int M = c->st.M, N = c->st.N;
    const int sseg = std::max(M, (N / 8 + M - 1) / M * M);
    const int nsseg = (N + sseg - 1) / sseg;
    KS_CUDA(c, c->stream_buf.ensure(size_t(N) * SM_COUNT * c->npad * sizeof(float)));
    if (c->geo64)
        k_stream<double><<<nblocks(c->npix * nsseg, 128), 128, 0, c->stream>>>(plan_view(c), c->st, c->npix, sseg, nsseg, c->stream_buf.as<float>());
    else
        k_stream<float><<<nblocks(c->npix * nsseg, 128), 128, 0, c->stream>>>(plan_view(c), c->st, c->npix, sseg, nsseg, c->stream_buf.as<float>());
    c->launches++;
    KS_CUDA(c, cudaGetLastError());
    return KS_OK;
}

constexpr int kCandRun = 16;   // samples per candidate mask (16 vs the whole segment: config 5 -28%, config 2 -3%)

template <int CH, int NT, int KM>
int launch_consume(ks_context* c, const MixedJob& job0, int ntot, int nsm, int per_sm) {
    MixedJob job = job0;
    const int N = c->st.N;
    constexpr int W = NT / 32;
    const size_t smem = MixedSmem<CH>::bytes(ntot, W, c->nkv);
    // split the sample range into segments until there are about eight work units per resident
    // warp, so that the most expensive unit is short
    const long long resident = (long long)nsm * per_sm * W;
    const long long base_units = job.nchunks * job.nframes * job.nvc;
    int nseg = 1;
    const int units_per_warp = c->tune_units > 0 ? c->tune_units : 8;
    while (job.nmax < 0 && base_units * nseg < units_per_warp * resident && (nseg * 2) * 16 <= N) nseg *= 2;
    job.seg_len = (N + nseg - 1) / nseg;
    job.nseg = (N + job.seg_len - 1) / job.seg_len;
    job.total = base_units * job.nseg;
    // candidate masks per run of samples (a segment's box spans the emission region in depth)
    job.cand_len = kCandRun;
    const double* dt = c->combos.as<double>();
    const double* dn = dt + job.nframes;
    job.gstate = c->fwd_gstate;
    job.gact = c->fwd_gact;
    c->last_job = job;
    const size_t seg_bytes = size_t(job.nframes) * job.nfreq * job.nseg * c->npix * 20 * sizeof(float);
    KS_CUDA(c, c->seg_out.ensure(seg_bytes));
    KS_CUDA(c, c->work.ensure(2 * sizeof(unsigned long long)));   // the adjoint's two counters: no move under a captured render
    KS_CUDA(c, cudaMemsetAsync(c->work.p, 0, sizeof(unsigned long long), c->stream));
    const long long grid = std::min<long long>(job.total / W + 1, (long long)nsm * per_sm);
    if (!c->capturing) cudaEventRecord(c->evc0, c->stream);
    k_consume<CH, NT, KM><<<unsigned(grid), NT, smem, c->stream>>>(
        plan_view(c), c->st, job, c->tab32.as<float>(), ntot, dt, dn, c->stream_buf.as<float>(), c->work.as<unsigned long long>(),
        c->seg_out.as<float>(), c->count_events ? c->counters.as<unsigned long long>() : nullptr, c->errflag.as<unsigned>());
    if (!c->capturing) {
        cudaEventRecord(c->evc1, c->stream);
        c->consume_timed = true;
    }
    c->launches++;
    c->kernel_launches++;
    KS_CUDA(c, cudaGetLastError());
    const long long nq = c->npix * (long long)job.nframes * job.nfreq;
    k_combine<<<nblocks(nq, 256), 256, 0, c->stream>>>(job, dn, c->seg_out.as<float>(), c->out_sorted.as<double>());
    c->launches++;
    KS_CUDA(c, cudaGetLastError());
    return KS_OK;
}

// Occupancy of k_consume<CH, NT, KM> with its shared memory for `ntot` splats (0 if it does not fit).
template <int CH, int NT, int KM>
int consume_blocks(ks_context* c, int ntot) {
    const size_t smem = MixedSmem<CH>::bytes(ntot, NT / 32, c->nkv);
    if (smem > 227 * 1024) return 0;
    if (cudaFuncSetAttribute(k_consume<CH, NT, KM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_consume<CH, NT, KM>, NT, smem) != cudaSuccess) { cudaGetLastError(); return 0; }
    return per_sm;
}

template <int CH, int KM>
int launch_mixed_ch(ks_context* c, int ntot, int nframes, int nfreq, double L, int nmax, double slab) {
    int nsm = 0;
    KS_CUDA(c, cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
    // 1. the FP32 sample stream (one march per ray, shared by every frame and frequency)
    {
        int s = launch_stream(c);
        if (s) return s;
    }
    MixedJob job;
    job.npix = c->npix; job.npad = c->npad; job.nframes = nframes; job.nfreq = nfreq;
    job.nvc = (nfreq + CH - 1) / CH;
    job.nchunks = (c->npix + 31) / 32;
    job.nmax = nmax; job.slab = float(slab); job.L = L;
    job.nkv = c->nkv;
    job.ch = CH;
    job.stage_test = c->stage_test;
    // the block size with the most resident warps (the per-warp shared memory sets the limit)
    const int w384 = consume_blocks<CH, 384, KM>(c, ntot) * 12, w256 = consume_blocks<CH, 256, KM>(c, ntot) * 8,
              w128 = consume_blocks<CH, 128, KM>(c, ntot) * 4;
    const int best = std::max(w384, std::max(w256, w128));
    if (best <= 0) return fail(c, KS_ERR_ARGUMENT, "too many splats for one launch (%d)", ntot);
    // the autotuner's block size when it fits
    if (c->tune_nt == 384 && w384 > 0) return launch_consume<CH, 384, KM>(c, job, ntot, nsm, w384 / 12);
    if (c->tune_nt == 256 && w256 > 0) return launch_consume<CH, 256, KM>(c, job, ntot, nsm, w256 / 8);
    if (c->tune_nt == 128 && w128 > 0) return launch_consume<CH, 128, KM>(c, job, ntot, nsm, w128 / 4);
    if (w384 == best) return launch_consume<CH, 384, KM>(c, job, ntot, nsm, w384 / 12);
    if (w256 == best) return launch_consume<CH, 256, KM>(c, job, ntot, nsm, w256 / 8);
    if (w128 > 0) return launch_consume<CH, 128, KM>(c, job, ntot, nsm, w128 / 4);
    return fail(c, KS_ERR_ARGUMENT, "too many splats for one launch (%d)", ntot);
}

// The most warps of k_consume<CH, *, KM> resident per SM for an ntot-splat table.
template <int CH, int KM>
int resident_warps(ks_context* c, int ntot) {
    return std::max(consume_blocks<CH, 384, KM>(c, ntot) * 12, std::max(consume_blocks<CH, 256, KM>(c, ntot) * 8,
                                                                        consume_blocks<CH, 128, KM>(c, ntot) * 4));
}

// The frequencies of a work unit: all of them (up to four) share the march and the splat tests,
// unless the per-thread states of four frequencies and a large splat table leave room for half as
// many warps as two frequencies per unit would: then two (every sample is tested twice, but with the
// block-cooperative consumer occupancy pays more: the 256-splat movie ran 4 warps per SM with four).
template <int KM>
int launch_mixed_km(ks_context* c, int ntot, int nframes, int nfreq, double L, int nmax, double slab) {
    if (nfreq >= 4) {
        if (resident_warps<2, KM>(c, ntot) >= 2 * resident_warps<4, KM>(c, ntot))
            return launch_mixed_ch<2, KM>(c, ntot, nframes, nfreq, L, nmax, slab);
        return launch_mixed_ch<4, KM>(c, ntot, nframes, nfreq, L, nmax, slab);
    }
    if (nfreq == 3) return launch_mixed_ch<3, KM>(c, ntot, nframes, nfreq, L, nmax, slab);
    if (nfreq == 2) return launch_mixed_ch<2, KM>(c, ntot, nframes, nfreq, L, nmax, slab);
    return launch_mixed_ch<1, KM>(c, ntot, nframes, nfreq, L, nmax, slab);
}

int launch_mixed(ks_context* c, int ntot, const double* ht, int nframes, int nfreq, double L, int nmax, double slab, bool thermal_only) {
    (void)ht;
    if (ntot > 32 * kMaxSplatWords) return fail(c, KS_ERR_ARGUMENT, "the mixed path takes at most %d splats (%d)", 32 * kMaxSplatWords, ntot);
    return thermal_only ? launch_mixed_km<1>(c, ntot, nframes, nfreq, L, nmax, slab) : launch_mixed_km<7>(c, ntot, nframes, nfreq, L, nmax, slab);
}

// Write `nvec` x npix x width doubles from the sorted device buffer to `out` (host or device) in `order`.
int emit(ks_context* c, const double* sorted, int width, int nvec, int order, double* out) {
    size_t bytes = size_t(c->npix) * width * nvec * sizeof(double);
    bool dev = is_device_ptr(out);
    double* dst = out;
    if (!dev) { KS_CUDA(c, c->stage_out.ensure(bytes)); dst = c->stage_out.as<double>(); }
    long long total = c->npix * nvec;
    k_unsort<<<nblocks(total), kBlock, 0, c->stream>>>(sorted, c->perm.as<long long>(), c->npix, width, nvec,
                                                       order == KS_ORDER_SCREEN ? 1 : 0, dst);
    c->launches++;
    KS_CUDA(c, cudaGetLastError());
    if (!dev) KS_CUDA(c, cudaMemcpyAsync(out, dst, bytes, cudaMemcpyDeviceToHost, c->stream));
    return KS_OK;
}

}  // namespace

// ---- C ABI -------------------------------------------------------------------------------------------

extern "C" {

int ks_context_create(int device, int flags, ks_context** out) {
    (void)flags;
    if (!out) return KS_ERR_ARGUMENT;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) { cudaGetLastError(); return KS_ERR_DEVICE; }
    if (cudaSetDevice(device) != cudaSuccess) return KS_ERR_DEVICE;
    ks_context* c = new ks_context();
    c->device = device;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) { delete c; return KS_ERR_DEVICE; }
    cudaEventCreate(&c->ev0);
    cudaEventCreate(&c->ev1);
    cudaEventCreate(&c->evc0);
    cudaEventCreate(&c->evc1);
    cudaEventCreate(&c->evg0);
    cudaEventCreate(&c->evg1);
    if (c->errflag.ensure(sizeof(unsigned)) != cudaSuccess || cudaMemset(c->errflag.p, 0, sizeof(unsigned)) != cudaSuccess) {
        delete c;
        return KS_ERR_DEVICE;
    }
    init_constants();
    if (cudaGetLastError() != cudaSuccess) { delete c; return KS_ERR_DEVICE; }
    *out = c;
    return KS_OK;
}

int ks_context_destroy(ks_context* c) {
    if (!c) return KS_OK;
    cudaSetDevice(c->device);
    for (DevBuf* b : {&c->alpha, &c->beta, &c->key, &c->key2, &c->idx, &c->perm, &c->plan, &c->nanch, &c->aoff, &c->anchors,
                      &c->resid_t, &c->resid_phi, &c->scratch, &c->tab, &c->combos, &c->out_sorted, &c->stage_in, &c->stage_out, &c->counters, &c->seg_out, &c->work, &c->stream_buf, &c->inv_perm, &c->dft_tu, &c->dft_tv,
                      &c->dft_a, &c->dft_t, &c->dft_c, &c->dft_s, &c->dft_partial})
        b->release();
    for (DevBuf& b : c->dft_in) b.release();
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->evc0) cudaEventDestroy(c->evc0);
    if (c->evc1) cudaEventDestroy(c->evc1);
    if (c->evg0) cudaEventDestroy(c->evg0);
    if (c->evg1) cudaEventDestroy(c->evg1);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
    if (c->graph) cudaGraphDestroy(c->graph);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return KS_OK;
}

const char* ks_last_error(const ks_context* c) { return c ? c->err.c_str() : "null context"; }

int ks_context_stream(ks_context* c, void** stream) {
    if (!c || !stream) return KS_ERR_ARGUMENT;
    *stream = (void*)c->stream;
    return KS_OK;
}

// Accumulated device time of the render kernels (k_thin / k_polarized) since the last reset, and
// the number of launches of this library's kernels.
int ks_kernel_stats(ks_context* c, double* render_ms, long long* render_launches, long long* all_launches, int reset) {
    if (!c) return KS_ERR_ARGUMENT;
    if (render_ms) *render_ms = c->kernel_ms;
    if (render_launches) *render_launches = c->kernel_launches;
    if (all_launches) *all_launches = c->launches;
    if (reset) { c->kernel_ms = 0.0; c->kernel_launches = 0; c->launches = 0; }
    return KS_OK;
}

// Test hook of the staging error path: while on, the mixed kernels arm their table-staging barrier
// without issuing the copy, so the bounded wait runs out and the call fails with KS_ERR_TIMEOUT.
int ks_set_stage_test(ks_context* c, int32_t on) {
    if (!c) return KS_ERR_ARGUMENT;
    c->stage_test = on ? 1 : 0;
    return KS_OK;
}

int ks_gemm_stats(ks_context* c, double* ms, long long* launches, double* flops, int reset) {
    if (!c) return KS_ERR_ARGUMENT;
    if (ms) *ms = c->gemm_ms;
    if (launches) *launches = c->gemm_launches;
    if (flops) *flops = c->gemm_flops;
    if (reset) { c->gemm_ms = 0.0; c->gemm_launches = 0; c->gemm_flops = 0.0; }
    return KS_OK;
}

int ks_set_tensor_path(ks_context* c, int32_t path) {
    if (!c) return KS_ERR_ARGUMENT;
    if (path != KS_TENSOR_TCGEN05 && path != KS_TENSOR_MMA_SYNC) return fail(c, KS_ERR_ARGUMENT, "unknown tensor path %d", path);
    c->tensor_path = path;
    return KS_OK;
}

// Device time of k_consume alone in the mixed ks_render calls since the last reset, and its launches.
int ks_consume_stats(ks_context* c, double* consume_ms, long long* launches, int reset) {
    if (!c) return KS_ERR_ARGUMENT;
    if (consume_ms) *consume_ms = c->consume_ms;
    if (launches) *launches = c->consume_launches;
    if (reset) { c->consume_ms = 0.0; c->consume_launches = 0; }
    return KS_OK;
}

// Count the work events of the following ks_render calls (samples, valid samples, splat tests,
// weights, coefficient evaluations, frames, steps) into a device counter; ks_event_counts reads them.
int ks_set_event_counting(ks_context* c, int on) {
    if (!c) return KS_ERR_ARGUMENT;
    c->count_events = on != 0;
    return KS_OK;
}

int ks_event_counts(ks_context* c, unsigned long long out[7]) {
    if (!c || !out) return KS_ERR_ARGUMENT;
    if (!c->counters.p) { for (int q = 0; q < 7; ++q) out[q] = 0; return KS_OK; }
    KS_CUDA(c, cudaMemcpy(out, c->counters.p, 7 * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    return KS_OK;
}

int ks_camera_set(ks_context* c, const double* alpha, const double* beta, int64_t npix, int32_t nalpha, int32_t nbeta) {
    if (!c) return KS_ERR_ARGUMENT;
    if (!alpha || !beta || npix <= 0) return fail(c, KS_ERR_ARGUMENT, "camera needs at least one pixel");
    if ((long long)nalpha * nbeta != npix) return fail(c, KS_ERR_ARGUMENT, "camera pixel vectors do not match the screen size");
    KS_CUDA(c, cudaSetDevice(c->device));
    std::vector<double> ha(npix), hb(npix);
    KS_CUDA(c, cudaMemcpy(ha.data(), alpha, npix * sizeof(double), cudaMemcpyDefault));
    KS_CUDA(c, cudaMemcpy(hb.data(), beta, npix * sizeof(double), cudaMemcpyDefault));
    for (long long i = 0; i < npix; ++i)
        if (!std::isfinite(ha[i]) || !std::isfinite(hb[i])) return fail(c, KS_ERR_NONFINITE, "non-finite screen coordinate at pixel %lld", i);
    c->npix = npix;
    c->npad = (npix + 31) / 32 * 32;
    c->nalpha = nalpha; c->nbeta = nbeta;
    KS_CUDA(c, c->alpha.ensure(npix * sizeof(double)));
    KS_CUDA(c, c->beta.ensure(npix * sizeof(double)));
    KS_CUDA(c, cudaMemcpy(c->alpha.p, ha.data(), npix * sizeof(double), cudaMemcpyHostToDevice));
    KS_CUDA(c, cudaMemcpy(c->beta.p, hb.data(), npix * sizeof(double), cudaMemcpyHostToDevice));
    c->regenerated = false;
    return KS_OK;
}

namespace {
int regenerate_impl(ks_context* c, double a, double theta_o, int32_t nsamples, int32_t anchor_M, double density, int32_t nmin);
}

int ks_regenerate(ks_context* c, double a, double theta_o, int32_t nsamples, int32_t anchor_M) {
    return regenerate_impl(c, a, theta_o, nsamples, anchor_M, 0.0, 0);
}

int ks_regenerate_uneven(ks_context* c, double a, double theta_o, double samples_per_mino, int32_t nmin, int32_t nmax, int32_t anchor_M) {
    if (!c) return KS_ERR_ARGUMENT;
    if (!(std::isfinite(samples_per_mino) && samples_per_mino > 0)) return fail(c, KS_ERR_ARGUMENT, "samples per unit Mino time must be positive");
    if (nmin < 1 || nmax < nmin) return fail(c, KS_ERR_ARGUMENT, "need 1 <= nmin <= nmax");
    return regenerate_impl(c, a, theta_o, nmax, anchor_M, samples_per_mino, nmin);
}

int ks_get_nsamples(ks_context* c, int32_t* out) {
    if (!c || !out) return KS_ERR_ARGUMENT;
    if (!c->regenerated) return fail(c, KS_ERR_NOT_REGENERATED, "regenerate the context first");
    std::vector<double> f(c->npix);
    KS_CUDA(c, cudaMemcpy(f.data(), c->plan.as<double>() + size_t(PF_NSAMP) * c->npad, c->npix * sizeof(double), cudaMemcpyDeviceToHost));
    std::vector<int32_t> o(c->npix);
    for (long long j = 0; j < c->npix; ++j) o[j] = int32_t(f[j]);
    KS_CUDA(c, cudaMemcpy(out, o.data(), o.size() * sizeof(int32_t), cudaMemcpyDefault));
    return KS_OK;
}

}  // extern "C"

namespace {
int regenerate_impl(ks_context* c, double a, double theta_o, int32_t nsamples, int32_t anchor_M, double density, int32_t nmin) {
    if (!c) return KS_ERR_ARGUMENT;
    if (c->npix <= 0) return fail(c, KS_ERR_ARGUMENT, "set a camera before regenerate");
    ks_graph_destroy(c);   // a captured render holds the old geometry's launch shape
    if (!std::isfinite(a) || !std::isfinite(theta_o)) return fail(c, KS_ERR_NONFINITE, "non-finite spin or inclination");
    if (!(a > 0.0 && a < 1.0)) return fail(c, KS_ERR_ARGUMENT, "spin must lie in (0, 1) (the analytic polar solution divides by a)");
    if (nsamples < 1) return fail(c, KS_ERR_ARGUMENT, "need at least one sample per ray");
    if (anchor_M < 1) return fail(c, KS_ERR_ARGUMENT, "re-anchoring interval must be positive");
    KS_CUDA(c, cudaSetDevice(c->device));
    const long long n = c->npix, npad = c->npad;
    Spacetime& st = c->st;
    st.a = a; st.thetao = theta_o;
    st.rp = 1.0 + std::sqrt(1.0 - a * a); st.rmn = 1.0 - std::sqrt(1.0 - a * a); st.rh = st.rp;
    st.abscos = std::fabs(std::cos(theta_o)); st.cos2 = std::cos(theta_o) * std::cos(theta_o);
    st.N = nsamples; st.M = anchor_M;
    st.density = density; st.nmin = nmin;
    KS_CUDA(c, c->key.ensure(n)); KS_CUDA(c, c->key2.ensure(n));
    KS_CUDA(c, c->idx.ensure(n * sizeof(long long))); KS_CUDA(c, c->perm.ensure(n * sizeof(long long)));
    k_root_case<<<nblocks(n), kBlock, 0, c->stream>>>(st, c->alpha.as<double>(), c->beta.as<double>(), n, c->key.as<unsigned char>(),
                                                        c->idx.as<long long>());
    c->launches++;
    KS_CUDA(c, cudaGetLastError());
    size_t tmp = 0;
    KS_CUDA(c, cub::DeviceRadixSort::SortPairs(nullptr, tmp, c->key.as<unsigned char>(), c->key2.as<unsigned char>(),
                                               c->idx.as<long long>(), c->perm.as<long long>(), (int)n, 0, 3, c->stream));
    KS_CUDA(c, c->scratch.ensure(tmp));
    KS_CUDA(c, cub::DeviceRadixSort::SortPairs(c->scratch.p, tmp, c->key.as<unsigned char>(), c->key2.as<unsigned char>(),
                                               c->idx.as<long long>(), c->perm.as<long long>(), (int)n, 0, 3, c->stream));
    KS_CUDA(c, c->plan.ensure(size_t(PF_COUNT) * npad * sizeof(double)));
    KS_CUDA(c, c->nanch.ensure(n * sizeof(long long)));
    KS_CUDA(c, c->aoff.ensure((n + 1) * sizeof(long long)));
    k_build_plan<<<nblocks(n), kBlock, 0, c->stream>>>(st, c->alpha.as<double>(), c->beta.as<double>(), c->perm.as<long long>(), n, npad,
                                                         c->plan.as<double>(), c->nanch.as<long long>());
    c->launches++;
    KS_CUDA(c, cudaGetLastError());
    tmp = 0;
    KS_CUDA(c, cub::DeviceScan::ExclusiveSum(nullptr, tmp, c->nanch.as<long long>(), c->aoff.as<long long>(), (int)n, c->stream));
    KS_CUDA(c, c->scratch.ensure(tmp));
    KS_CUDA(c, cub::DeviceScan::ExclusiveSum(c->scratch.p, tmp, c->nanch.as<long long>(), c->aoff.as<long long>(), (int)n, c->stream));
    // totals and case ranges
    std::vector<long long> hn(n), ho(n);
    std::vector<unsigned char> hk(n);
    KS_CUDA(c, cudaMemcpyAsync(hn.data(), c->nanch.p, n * sizeof(long long), cudaMemcpyDeviceToHost, c->stream));
    KS_CUDA(c, cudaMemcpyAsync(ho.data(), c->aoff.p, n * sizeof(long long), cudaMemcpyDeviceToHost, c->stream));
    KS_CUDA(c, cudaMemcpyAsync(hk.data(), c->key2.p, n, cudaMemcpyDeviceToHost, c->stream));
    KS_CUDA(c, cudaStreamSynchronize(c->stream));
    c->total_anchors = ho[n - 1] + hn[n - 1];
    c->max_nanch = 0;
    for (long long j = 0; j < n; ++j) c->max_nanch = std::max<int>(c->max_nanch, (int)hn[j]);
    long long cnt[3] = {0, 0, 0};
    for (long long j = 0; j < n; ++j) cnt[hk[j] / 2]++;
    c->ranges[0] = 0; c->ranges[1] = cnt[0];
    c->ranges[2] = cnt[0]; c->ranges[3] = cnt[0] + cnt[1];
    c->ranges[4] = cnt[0] + cnt[1]; c->ranges[5] = n;
    KS_CUDA(c, c->anchors.ensure(size_t(c->total_anchors) * AF_COUNT * sizeof(double)));
    dim3 grid(nblocks(n), c->max_nanch);
    k_anchor_segments<<<grid, kBlock, 0, c->stream>>>(st, c->alpha.as<double>(), c->beta.as<double>(), c->perm.as<long long>(), n, npad,
                                                       c->plan.as<double>(), c->aoff.as<long long>(), c->anchors.as<double>());
    c->launches++;
    KS_CUDA(c, cudaGetLastError());
    k_anchor_prefix<<<nblocks(n), kBlock, 0, c->stream>>>(n, npad, c->plan.as<double>(), c->aoff.as<long long>(), c->anchors.as<double>());
    c->launches++;
    KS_CUDA(c, cudaGetLastError());
    KS_CUDA(c, c->inv_perm.ensure(n * sizeof(long long)));
    k_inverse_perm<<<nblocks(n), kBlock, 0, c->stream>>>(c->perm.as<long long>(), n, c->inv_perm.as<long long>());
    c->launches++;
    KS_CUDA(c, cudaGetLastError());
    KS_CUDA(c, c->resid_t.ensure(n * sizeof(double)));
    KS_CUDA(c, c->resid_phi.ensure(n * sizeof(double)));
    KS_CUDA(c, cudaMemsetAsync(c->resid_t.p, 0, n * sizeof(double), c->stream));
    KS_CUDA(c, cudaMemsetAsync(c->resid_phi.p, 0, n * sizeof(double), c->stream));
    KS_CUDA(c, cudaStreamSynchronize(c->stream));
    c->regenerated = true;
    c->samples_ready = false;
    return KS_OK;
}
}  // namespace

extern "C" {

int ks_get_perm(ks_context* c, int64_t* perm) {
    if (!c || !perm) return KS_ERR_ARGUMENT;
    if (!c->regenerated) return fail(c, KS_ERR_NOT_REGENERATED, "regenerate the context first");
    KS_CUDA(c, cudaMemcpy(perm, c->perm.p, c->npix * sizeof(long long), cudaMemcpyDefault));
    return KS_OK;
}

int ks_get_ranges(ks_context* c, int64_t ranges[6]) {
    if (!c || !ranges) return KS_ERR_ARGUMENT;
    if (!c->regenerated) return fail(c, KS_ERR_NOT_REGENERATED, "regenerate the context first");
    for (int q = 0; q < 6; ++q) ranges[q] = c->ranges[q];
    return KS_OK;
}

int ks_get_residuals(ks_context* c, double* rt, double* rp) {
    if (!c || !rt || !rp) return KS_ERR_ARGUMENT;
    if (!c->regenerated) return fail(c, KS_ERR_NOT_REGENERATED, "regenerate the context first");
    KS_CUDA(c, cudaMemcpy(rt, c->resid_t.p, c->npix * sizeof(double), cudaMemcpyDefault));
    KS_CUDA(c, cudaMemcpy(rp, c->resid_phi.p, c->npix * sizeof(double), cudaMemcpyDefault));
    return KS_OK;
}

int ks_get_ray_constants(ks_context* c, double* out) {
    if (!c || !out) return KS_ERR_ARGUMENT;
    if (!c->regenerated) return fail(c, KS_ERR_NOT_REGENERATED, "regenerate the context first");
    const long long n = c->npix, np = c->npad;
    std::vector<double> f(size_t(PF_COUNT) * np);
    KS_CUDA(c, cudaMemcpy(f.data(), c->plan.p, f.size() * sizeof(double), cudaMemcpyDeviceToHost));
    std::vector<double> o(size_t(n) * 24);
    const int fields[24] = {PF_ETA, PF_LAM, PF_NUMREALS, PF_K, PF_C, PF_FO, PF_TAU_TOTAL, PF_TAU_VALID, PF_GTHO,
                            PF_R1RE, PF_R1IM, PF_R2RE, PF_R2IM, PF_R3RE, PF_R3IM, PF_R4RE, PF_R4IM,
                            PF_PMU, PF_PSCALE, PF_TEMPFAC, PF_POFFSET, PF_MANCHOR, PF_K2, PF_SCATTER};
    for (long long j = 0; j < n; ++j)
        for (int q = 0; q < 24; ++q) o[size_t(j) * 24 + q] = f[size_t(fields[q]) * np + j];
    KS_CUDA(c, cudaMemcpy(out, o.data(), o.size() * sizeof(double), cudaMemcpyDefault));
    return KS_OK;
}

int ks_march_samples(ks_context* c, double* t, double* r, double* theta, double* phi, uint8_t* flags) {
    if (!c || !t || !r || !theta || !phi || !flags) return KS_ERR_ARGUMENT;
    if (!c->regenerated) return fail(c, KS_ERR_NOT_REGENERATED, "regenerate the context first");
    KS_CUDA(c, cudaSetDevice(c->device));
    const long long n = c->npix;
    const size_t ns = size_t(n) * c->st.N;
    KS_CUDA(c, c->stage_out.ensure(ns * (4 * sizeof(double) + 1)));
    double* d = c->stage_out.as<double>();
    unsigned char* fl = reinterpret_cast<unsigned char*>(d + 4 * ns);
    KS_CUDA(c, cudaMemsetAsync(d, 0, ns * (4 * sizeof(double) + 1), c->stream));   // samples past a ray's count: zero
    k_march_store<<<nblocks(n), kBlock, 0, c->stream>>>(plan_view(c), c->st, n, d, d + ns, d + 2 * ns, d + 3 * ns, fl,
                                                          c->resid_t.as<double>(), c->resid_phi.as<double>());
    c->launches++;
    KS_CUDA(c, cudaGetLastError());
    KS_CUDA(c, cudaMemcpyAsync(t, d, ns * sizeof(double), cudaMemcpyDefault, c->stream));
    KS_CUDA(c, cudaMemcpyAsync(r, d + ns, ns * sizeof(double), cudaMemcpyDefault, c->stream));
    KS_CUDA(c, cudaMemcpyAsync(theta, d + 2 * ns, ns * sizeof(double), cudaMemcpyDefault, c->stream));
    KS_CUDA(c, cudaMemcpyAsync(phi, d + 3 * ns, ns * sizeof(double), cudaMemcpyDefault, c->stream));
    KS_CUDA(c, cudaMemcpyAsync(flags, fl, ns, cudaMemcpyDefault, c->stream));
    KS_CUDA(c, cudaStreamSynchronize(c->stream));
    return KS_OK;
}

int ks_thin_image(ks_context* c, const double* params, int32_t nsplat, double t_obs, int32_t precision, double* out, int32_t order) {
    if (!c || !out) return KS_ERR_ARGUMENT;
    if (!c->regenerated) return fail(c, KS_ERR_NOT_REGENERATED, "regenerate the context first");
    if (nsplat < 0 || (nsplat > 0 && !params)) return fail(c, KS_ERR_ARGUMENT, "bad splat count or parameters");
    if (precision != KS_FP64 && precision != KS_MIXED) return fail(c, KS_ERR_ARGUMENT, "unknown precision %d", precision);
    if (order != KS_ORDER_SORTED && order != KS_ORDER_SCREEN) return fail(c, KS_ERR_ARGUMENT, "unknown order %d", order);
    if (!std::isfinite(t_obs)) return fail(c, KS_ERR_NONFINITE, "non-finite observation time");
    KS_CUDA(c, cudaSetDevice(c->device));
    const long long n = c->npix;
    const void* dparams = nullptr;
    if (nsplat > 0) {
        int s = stage_in(c, c->stage_in, params, size_t(14) * nsplat * sizeof(double), &dparams);
        if (s) return s;
    }
    KS_CUDA(c, c->tab.ensure(size_t(std::max(nsplat, 1)) * ST_COUNT * sizeof(double)));
    if (nsplat > 0) {
        SetDesc d{KS_THIN14, 14, nsplat, 0, (const double*)dparams, nullptr, 0.0};
        k_splat_table<<<nblocks(nsplat, 64), 64, 0, c->stream>>>(d, c->tab.as<double>());
        c->launches++;
        KS_CUDA(c, cudaGetLastError());
    }
    KS_CUDA(c, c->out_sorted.ensure(n * sizeof(double)));
    size_t smem = size_t(nsplat) * ST_COUNT * (precision == KS_FP64 ? sizeof(double) : sizeof(float));
    if (smem > 200 * 1024) return fail(c, KS_ERR_ARGUMENT, "too many splats for one launch (%d)", nsplat);
    cudaEventRecord(c->ev0, c->stream);
    if (precision == KS_FP64) {
        KS_CUDA(c, cudaFuncSetAttribute(k_thin<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_thin<double><<<nblocks(n), kBlock, smem, c->stream>>>(plan_view(c), c->st, n, c->tab.as<double>(), nsplat, t_obs, nullptr,
                                                                 c->out_sorted.as<double>(), c->resid_t.as<double>(), c->resid_phi.as<double>());
    } else {
        KS_CUDA(c, cudaFuncSetAttribute(k_thin<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_thin<float><<<nblocks(n), kBlock, smem, c->stream>>>(plan_view(c), c->st, n, c->tab.as<double>(), nsplat, t_obs, nullptr,
                                                                c->out_sorted.as<double>(), nullptr, nullptr);
    }
    cudaEventRecord(c->ev1, c->stream);
    c->launches++;
    KS_CUDA(c, cudaGetLastError());
    int s = emit(c, c->out_sorted.as<double>(), 1, 1, order, out);
    if (s) return s;
    KS_CUDA(c, cudaStreamSynchronize(c->stream));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    c->kernel_ms += ms; c->kernel_launches++;
    return KS_OK;
}

int ks_render(ks_context* c, const ks_splat_set* sets, int32_t nsets, const double* times, int32_t nframes, const double* nus,
              int32_t nfreq, double L, int32_t precision, int32_t nmax, double slab, double* out, int32_t order) {
    if (!c || !out) return KS_ERR_ARGUMENT;
    if (!c->regenerated) return fail(c, KS_ERR_NOT_REGENERATED, "regenerate the context first");
    if (nsets < 0 || (nsets > 0 && !sets)) return fail(c, KS_ERR_ARGUMENT, "bad splat sets");
    if (nframes < 1 || nfreq < 1 || !times || !nus) return fail(c, KS_ERR_ARGUMENT, "need at least one frame and one frequency");
    if (precision != KS_FP64 && precision != KS_MIXED && precision != KS_MIXED_GEO64)
        return fail(c, KS_ERR_ARGUMENT, "unknown precision %d", precision);
    if (order != KS_ORDER_SORTED && order != KS_ORDER_SCREEN) return fail(c, KS_ERR_ARGUMENT, "unknown order %d", order);
    if (!(std::isfinite(L) && L > 0)) return fail(c, KS_ERR_NONFINITE, "length unit must be finite and positive");
    c->geo64 = precision == KS_MIXED_GEO64;
    if (precision == KS_MIXED_GEO64) precision = KS_MIXED;
    if (!std::isfinite(slab)) return fail(c, KS_ERR_NONFINITE, "non-finite slab");
    KS_CUDA(c, cudaSetDevice(c->device));
    std::vector<double> ht(nframes), hnu(nfreq);
    KS_CUDA(c, cudaMemcpy(ht.data(), times, nframes * sizeof(double), cudaMemcpyDefault));
    KS_CUDA(c, cudaMemcpy(hnu.data(), nus, nfreq * sizeof(double), cudaMemcpyDefault));
    for (double v : ht) if (!std::isfinite(v)) return fail(c, KS_ERR_NONFINITE, "non-finite observation time");
    for (double v : hnu) if (!(std::isfinite(v) && v > 0)) return fail(c, KS_ERR_NONFINITE, "frequencies must be finite and positive");
    int ntot = 0;
    {
        int st_ = build_tables(c, sets, nsets, &ntot, false);
        if (st_) return st_;
    }
    const long long n = c->npix;
    const int ncombo = nframes * nfreq;
    std::vector<double> hc(2 * size_t(ncombo));
    for (int fv = 0; fv < nfreq; ++fv)
        for (int ft = 0; ft < nframes; ++ft) {
            hc[size_t(fv) * nframes + ft] = ht[ft];
            hc[ncombo + size_t(fv) * nframes + ft] = hnu[fv];
        }
    if (precision == KS_MIXED) {
        // times then frequencies
        hc.assign(ht.begin(), ht.end());
        hc.insert(hc.end(), hnu.begin(), hnu.end());
    }
    // sized for the adjoint's layout too (times, frequencies, then per combination), so that an
    // adjoint call does not move the buffer under a captured render
    KS_CUDA(c, c->combos.ensure((size_t(nframes) + nfreq + 2 * size_t(ncombo)) * sizeof(double)));
    KS_CUDA(c, cudaMemcpyAsync(c->combos.p, hc.data(), hc.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    KS_CUDA(c, c->out_sorted.ensure(size_t(n) * 4 * ncombo * sizeof(double)));
    const double* dct = c->combos.as<double>();
    const double* dcn = dct + ncombo;
    if (c->count_events) {
        KS_CUDA(c, c->counters.ensure(8 * sizeof(unsigned long long)));
        KS_CUDA(c, cudaMemsetAsync(c->counters.p, 0, 8 * sizeof(unsigned long long), c->stream));
    }
    cudaEventRecord(c->ev0, c->stream);
    if (precision == KS_FP64) {
        // the plain path: one march per (frame, frequency), as the reference's polarized_cube does
        size_t smem = (size_t(ntot) * ST_COUNT + c->nkv) * sizeof(double);
        if (smem > 220 * 1024) return fail(c, KS_ERR_ARGUMENT, "too many splats for one launch (%d)", ntot);
        KS_CUDA(c, cudaFuncSetAttribute(k_polarized<double, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        for (int cc = 0; cc < ncombo; ++cc) {
            k_polarized<double, 1><<<dim3(nblocks(n), 1), kBlock, smem, c->stream>>>(
                plan_view(c), c->st, n, c->tab.as<double>(), ntot, dct + cc, dcn + cc, 1, L, nmax, slab,
                c->out_sorted.as<double>() + size_t(cc) * n * 4, c->resid_t.as<double>(), c->resid_phi.as<double>(),
                c->count_events ? c->counters.as<unsigned long long>() : nullptr, c->nkv);
            c->launches++;
            c->kernel_launches++;
        }
    } else {
        // the mixed path: one launch over rays x (frame, frequency chunk)
        bool thermal_only = true;
        for (int q = 0; q < nsets; ++q) thermal_only = thermal_only && (sets[q].kind == KS_THERMAL21 || sets[q].nsplat == 0);
        int s = launch_mixed(c, ntot, ht.data(), nframes, nfreq, L, nmax, slab, thermal_only);
        if (s) return s;
    }
    cudaEventRecord(c->ev1, c->stream);
    KS_CUDA(c, cudaGetLastError());
    int s = emit(c, c->out_sorted.as<double>(), 4, ncombo, order, out);
    if (s) return s;
    KS_CUDA(c, cudaStreamSynchronize(c->stream));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    c->kernel_ms += ms;
    if (precision != KS_FP64 && c->consume_timed) {
        float mc = 0.f;
        cudaEventElapsedTime(&mc, c->evc0, c->evc1);
        c->consume_ms += mc;
        c->consume_launches++;
        c->consume_timed = false;
    }
    if (precision != KS_FP64) return check_device_flag(c, "ks_render");
    return KS_OK;
}

int ks_riaf_image(ks_context* c, const double* model, int32_t pandya, const double* nus, int32_t nfreq, double L, int32_t precision,
                  double* out, int32_t order) {
    if (!c || !out || !model || !nus) return KS_ERR_ARGUMENT;
    if (!c->regenerated) return fail(c, KS_ERR_NOT_REGENERATED, "regenerate the context first");
    if (nfreq < 1) return fail(c, KS_ERR_ARGUMENT, "need at least one frequency");
    if (precision != KS_FP64 && precision != KS_MIXED) return fail(c, KS_ERR_ARGUMENT, "unknown precision %d", precision);
    if (order != KS_ORDER_SORTED && order != KS_ORDER_SCREEN) return fail(c, KS_ERR_ARGUMENT, "unknown order %d", order);
    if (!(std::isfinite(L) && L > 0)) return fail(c, KS_ERR_NONFINITE, "length unit must be finite and positive");
    KS_CUDA(c, cudaSetDevice(c->device));
    double hm[KS_RIAF_PARAMS];
    KS_CUDA(c, cudaMemcpy(hm, model, sizeof hm, cudaMemcpyDefault));
    for (double v : hm) if (!std::isfinite(v)) return fail(c, KS_ERR_NONFINITE, "non-finite RIAF parameter");
    if (!(hm[9] > 0 && hm[8] > 0 && hm[2] > 0)) return fail(c, KS_ERR_ARGUMENT, "RIAF needs positive disk_h, r_isco and rout");
    std::vector<double> hnu(nfreq);
    KS_CUDA(c, cudaMemcpy(hnu.data(), nus, nfreq * sizeof(double), cudaMemcpyDefault));
    for (double v : hnu) if (!(std::isfinite(v) && v > 0)) return fail(c, KS_ERR_NONFINITE, "frequencies must be finite and positive");
    const RiafModel m{hm[0], hm[1], hm[2], hm[3], hm[4], hm[5], hm[6], hm[7], hm[8], hm[9], pandya != 0};
    const long long n = c->npix;
    KS_CUDA(c, c->combos.ensure(hnu.size() * sizeof(double)));
    KS_CUDA(c, cudaMemcpyAsync(c->combos.p, hnu.data(), hnu.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    KS_CUDA(c, c->out_sorted.ensure(size_t(n) * 4 * nfreq * sizeof(double)));
    if (c->count_events) {
        KS_CUDA(c, c->counters.ensure(8 * sizeof(unsigned long long)));
        KS_CUDA(c, cudaMemsetAsync(c->counters.p, 0, 8 * sizeof(unsigned long long), c->stream));
    }
    unsigned long long* ctr = c->count_events ? c->counters.as<unsigned long long>() : nullptr;
    cudaEventRecord(c->ev0, c->stream);
    const dim3 grid(unsigned(nblocks(n)), unsigned(nfreq));
    if (precision == KS_FP64)
        k_riaf<double><<<grid, kBlock, 0, c->stream>>>(plan_view(c), c->st, n, m, c->combos.as<double>(), L, c->out_sorted.as<double>(), ctr);
    else
        k_riaf<float><<<grid, kBlock, 0, c->stream>>>(plan_view(c), c->st, n, m, c->combos.as<double>(), L, c->out_sorted.as<double>(), ctr);
    cudaEventRecord(c->ev1, c->stream);
    c->launches++;
    c->kernel_launches++;
    KS_CUDA(c, cudaGetLastError());
    int s = emit(c, c->out_sorted.as<double>(), 4, nfreq, order, out);
    if (s) return s;
    KS_CUDA(c, cudaStreamSynchronize(c->stream));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    c->kernel_ms += ms;
    return KS_OK;
}

// The device buffers a captured render reads or writes (a replay requires them unmoved).
std::vector<void*> graph_buffers(const ks_context* c) {
    return {c->tab.p, c->tab32.p, c->stream_buf.p, c->seg_out.p, c->work.p, c->out_sorted.p, c->combos.p, c->errflag.p,
            c->perm.p, c->plan.p, c->anchors.p, c->aoff.p};
}

void release_graph(cudaGraph_t& g, cudaGraphExec_t& ex) {
    if (ex) cudaGraphExecDestroy(ex);
    if (g) cudaGraphDestroy(g);
    ex = nullptr;
    g = nullptr;
}

// ... and those of a captured chi^2 + gradient evaluation
std::vector<void*> chi2_graph_buffers(const ks_context* c) {
    std::vector<void*> b = graph_buffers(c);
    for (const DevBuf* d : {&c->gtab, &c->adj_state, &c->adj_act, &c->adj_bnd, &c->adj_unit, &c->adj_part, &c->seeds, &c->chi_part,
                            &c->chi_val, &c->dgrad})
        b.push_back(d->p);
    return b;
}

// The splat tables of device-resident sets rebuilt on the device inside a capture (the knot array
// stays as the ordinary call before the capture wrote it): k_splat_table per set, with grad the
// gradient table (k_grad_table), and the FP32 copy.
int capture_tables(ks_context* c, const ks_splat_set* sets, int nsets, int ntot, bool grad) {
    int first = 0, koff = 0;
    for (int s = 0; s < nsets; ++s) {
        const ks_splat_set& S = sets[s];
        if (S.nsplat == 0) continue;
        const int nk = S.kind == KS_KNOT21 ? S.nknots : 0;
        SetDesc d{S.kind, nrows_of(S.kind), S.nsplat, first, static_cast<const double*>(S.params),
                  S.kind == KS_KAPPA22 ? static_cast<const double*>(S.hyp) : nullptr, S.gamma_max > 0 ? S.gamma_max : 1e5,
                  S.kind == KS_KNOT21 ? koff : 0, nk,
                  c->tab.as<const double>() + size_t(ntot) * ST_COUNT};
        k_splat_table<<<nblocks(S.nsplat, 64), 64, 0, c->stream>>>(d, c->tab.as<double>());
        if (grad) k_grad_table<<<nblocks(S.nsplat, 64), 64, 0, c->stream>>>(S.nsplat, first, static_cast<const double*>(S.params),
                                                                           c->gtab.as<double>());
        if (cudaGetLastError() != cudaSuccess) return fail(c, KS_ERR_DEVICE, "graph capture: splat table of set %d", s);
        first += S.nsplat;
        koff += S.nsplat * 4 * nk;   // per knot splat: its nk times and 3 nk centres
    }
    const long long nv = (long long)ntot * ST_COUNT + c->nkv;
    const long long np4 = std::max<long long>(4, (nv + 3) / 4 * 4);
    k_tab_f32<<<nblocks(np4, 256), 256, 0, c->stream>>>(nv, np4, c->tab.as<double>(), c->tab32.as<float>());
    if (cudaGetLastError() != cudaSuccess) return fail(c, KS_ERR_DEVICE, "graph capture: FP32 table");
    return KS_OK;
}

// One mixed render of device-resident splat sets recorded into a CUDA graph: the splat tables built
// from the parameters (in place on the device), their FP32 copy, the sample stream, the consumer, the
// segment composition and the output in `order`. Frames, frequencies, L, the knot array, the splat
// counts and the pointers are fixed at capture; a replay re-reads the parameter values.
int ks_render_graph_capture(ks_context* c, const ks_splat_set* sets, int32_t nsets, const double* times, int32_t nframes,
                            const double* nus, int32_t nfreq, double L, int32_t nmax, double slab, double* out, int32_t order) {
    if (!c || !out || !sets || nsets < 1) return KS_ERR_ARGUMENT;
    if (!is_device_ptr(out)) return fail(c, KS_ERR_ARGUMENT, "the graph's output must be device memory");
    for (int s = 0; s < nsets; ++s) {
        if (sets[s].nsplat > 0 && !is_device_ptr(sets[s].params))
            return fail(c, KS_ERR_ARGUMENT, "set %d: a graph reads device-resident parameters", s);
        if (sets[s].kind == KS_KAPPA22 && sets[s].nsplat > 0 && !is_device_ptr(sets[s].hyp))
            return fail(c, KS_ERR_ARGUMENT, "set %d: a graph reads device-resident hyp", s);
    }
    release_graph(c->graph, c->graph_exec);
    const bool counting = c->count_events;
    c->count_events = false;
    // one ordinary render: validation, tables and knots, buffers, the launch shape
    int status = ks_render(c, sets, nsets, times, nframes, nus, nfreq, L, KS_MIXED, nmax, slab, out, order);
    c->count_events = counting;
    if (status) return status;
    int ntot = 0;
    bool thermal_only = true;
    for (int s = 0; s < nsets; ++s) {
        ntot += sets[s].nsplat;
        thermal_only = thermal_only && (sets[s].kind == KS_THERMAL21 || sets[s].nsplat == 0);
    }
    KS_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed));
    c->capturing = true;
    status = capture_tables(c, sets, nsets, ntot, false);
    if (status == KS_OK) status = launch_mixed(c, ntot, nullptr, nframes, nfreq, L, nmax, slab, thermal_only);
    if (status == KS_OK) status = emit(c, c->out_sorted.as<double>(), 4, nframes * nfreq, order, out);
    cudaGraph_t g = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(c->stream, &g);
    c->capturing = false;
    if (status != KS_OK || ec != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return status != KS_OK ? status : fail(c, KS_ERR_DEVICE, "graph capture: %s", cudaGetErrorString(ec));
    }
    cudaGraphExec_t ex = nullptr;
    const cudaError_t ei = cudaGraphInstantiate(&ex, g, 0);
    if (ei != cudaSuccess) {
        cudaGraphDestroy(g);
        cudaGetLastError();
        return fail(c, KS_ERR_DEVICE, "graph instantiation: %s", cudaGetErrorString(ei));
    }
    c->graph = g;
    c->graph_exec = ex;
    c->graph_bufs = graph_buffers(c);
    return KS_OK;
}

// Replay the captured render on the context stream; with wait, synchronise and report a kernel whose
// bounded wait gave up.
int ks_graph_launch(ks_context* c, int32_t wait) {
    if (!c) return KS_ERR_ARGUMENT;
    if (!c->graph_exec) return fail(c, KS_ERR_ARGUMENT, "no captured graph");
    if (graph_buffers(c) != c->graph_bufs)
        return fail(c, KS_ERR_ARGUMENT, "a later call reallocated buffers the graph uses: capture again");
    KS_CUDA(c, cudaGraphLaunch(c->graph_exec, c->stream));
    c->launches++;
    if (!wait) return KS_OK;
    KS_CUDA(c, cudaStreamSynchronize(c->stream));
    return check_device_flag(c, "graph replay");
}

int ks_graph_destroy(ks_context* c) {
    if (!c) return KS_ERR_ARGUMENT;
    release_graph(c->graph, c->graph_exec);
    release_graph(c->cgraph, c->cgraph_exec);
    return KS_OK;
}

}  // extern "C"

// ---- the adjoint (src/Splats/dual_gradient.jl, src/Fit/Fit.jl:451-577) --------------------------------

namespace {
int gemm(ks_context* c, int M, int N, int K, const float* Ah, const float* Al, long long lda, const float* Bh, const float* Bl, long long ldb,
         float* C, long long ldc);
int dft_stage(ks_context* c, int slot, const double* src, size_t count, const double** dev);
int dft_checks(ks_context* c, int64_t nuv, double psize, double scale, int32_t precision);
int dft_forward(ks_context* c, const double* dimg, int32_t order, int64_t nuv, const double* du, const double* dv, const double* dtap,
                double psize, double scale, int32_t precision, double* dV);
int dft_adjoint(ks_context* c, const double* dw, int64_t nuv, const double* du, const double* dv, const double* dtap, double psize,
                double scale, int32_t precision, double* dseed, int32_t order, bool have_twiddles);

// The visibility data of a frame (frame_chi2_seed!, device_visibilities.jl:97-111): nuv baselines,
// the gains g (complex, may be NULL), the data vis and sigma per Stokes; all host or device.
struct VisData {
    int64_t nuv;
    const double *u, *v, *tap, *g, *vis, *sigma;
    double psize, scale;
};
}

namespace {

__global__ void k_accumulate(double* __restrict__ dst, const double* __restrict__ src, long long n, int accumulate) {
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q < n) dst[q] = (accumulate ? dst[q] : 0.0) + src[q];
}

// The stored FP64 samples of every ray (the reference's store_samples cache, built once per regenerate).
int ensure_samples(ks_context* c, StoredSamples* S) {
    const long long n = c->npix;
    const size_t ns = size_t(n) * c->st.N;
    KS_CUDA(c, c->samples.ensure(ns * (4 * sizeof(double) + 1)));
    double* d = c->samples.as<double>();
    unsigned char* fl = reinterpret_cast<unsigned char*>(d + 4 * ns);
    if (!c->samples_ready) {
        KS_CUDA(c, cudaMemsetAsync(fl, 0, ns, c->stream));   // samples past a ray's count stay invalid
        k_march_store<<<nblocks(n), kBlock, 0, c->stream>>>(plan_view(c), c->st, n, d, d + ns, d + 2 * ns, d + 3 * ns, fl,
                                                              c->resid_t.as<double>(), c->resid_phi.as<double>());
        c->launches++;
        KS_CUDA(c, cudaGetLastError());
        c->samples_ready = true;
    }
    *S = StoredSamples{d, d + ns, d + 2 * ns, d + 3 * ns, fl};
    return KS_OK;
}

// Stage `count` elements of `src` (host or device) into `buf`; returns the device pointer.
template <class U>
int stage_dev(ks_context* c, DevBuf& buf, const U* src, size_t count, const U** dev) {
    if (!src) { *dev = nullptr; return KS_OK; }
    const void* d = nullptr;
    int s = stage_in(c, buf, src, count * sizeof(U), &d);
    *dev = reinterpret_cast<const U*>(d);
    return s;
}

// Occupancy of k_adj_elements<CH, NT> with its shared memory for `ntot` splats (0 if it does not fit).
template <int CH, int NT>
int adjoint_blocks(ks_context* c, int ntot, bool global_acc) {
    const size_t smem = AdjSmem<CH>::bytes(ntot, NT / 32, global_acc);
    if (smem > 227 * 1024) return 0;
    if (cudaFuncSetAttribute(k_adj_elements<CH, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_adj_elements<CH, NT>, NT, smem) != cudaSuccess) { cudaGetLastError(); return 0; }
    return per_sm;
}

template <int CH, int NT>
int launch_adjoint_mixed_nt(ks_context* c, int ntot, int per_sm, const double* dt, const double* dn, bool global_acc) {
    int nsm = 0;
    KS_CUDA(c, cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
    const MixedJob& job = c->last_job;
    const long long ncombo = (long long)job.nframes * job.nfreq;
    KS_CUDA(c, c->adj_bnd.ensure(size_t(ncombo) * job.nseg * 8 * c->npix * sizeof(float)));
    k_adj_bounds<<<nblocks(c->npix * ncombo, 256), 256, 0, c->stream>>>(job, dn, c->seg_out.as<float>(), c->seeds.as<double>(),
                                                                        c->adj_bnd.as<float>());
    c->launches++;
    KS_CUDA(c, cudaGetLastError());
    const long long gsz = (long long)ntot * GR_COUNT;
    KS_CUDA(c, c->adj_unit.ensure(size_t(job.total) * gsz * sizeof(float)));
    KS_CUDA(c, c->work.ensure(2 * sizeof(unsigned long long)));
    KS_CUDA(c, cudaMemsetAsync(c->work.p, 0, 2 * sizeof(unsigned long long), c->stream));
    // the step phase
    {
        constexpr int NS = 256, WS = NS / 32;
        const size_t smem = AdjSmem<CH>::step_bytes(WS);
        KS_CUDA(c, cudaFuncSetAttribute(k_adj_steps<CH, NS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per = 0;
        KS_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_adj_steps<CH, NS>, NS, smem));
        const long long grid = std::min<long long>(job.total / WS + 1, (long long)nsm * std::max(per, 1));
        k_adj_steps<CH, NS><<<unsigned(grid), NS, smem, c->stream>>>(c->st, job, dn, c->plan.as<double>(), c->stream_buf.as<float>(),
                                                                    job.gstate, job.gact, c->adj_bnd.as<float>(), c->work.as<unsigned long long>());
        c->launches++;
        c->adjoint_launches++;
        KS_CUDA(c, cudaGetLastError());
    }
    // the element phase
    {
        constexpr int W = NT / 32;
        const long long grid = std::min<long long>(job.total / W + 1, (long long)nsm * per_sm);
        const size_t smem = AdjSmem<CH>::bytes(ntot, W, global_acc);
        k_adj_elements<CH, NT><<<unsigned(grid), NT, smem, c->stream>>>(c->st, job, c->tab32.as<float>(), c->gtab.as<double>(), ntot, dt, dn,
                                                                       c->plan.as<double>(), c->stream_buf.as<float>(), job.gstate, job.gact,
                                                                       c->work.as<unsigned long long>() + 1, c->adj_unit.as<float>(),
                                                                       global_acc ? 1 : 0, c->errflag.as<unsigned>());
        c->launches++;
        c->adjoint_launches++;
        KS_CUDA(c, cudaGetLastError());
    }
    const int per_chunk = 256;
    const int nchunks = int((job.total + per_chunk - 1) / per_chunk);
    KS_CUDA(c, c->adj_part.ensure(size_t(nchunks) * gsz * sizeof(double)));
    k_unit_reduce1<<<dim3(nblocks(gsz, 128), nchunks), 128, 0, c->stream>>>(c->adj_unit.as<float>(), job.total, gsz, per_chunk,
                                                                             c->adj_part.as<double>());
    k_unit_reduce2<<<nblocks(gsz, 128), 128, 0, c->stream>>>(c->adj_part.as<double>(), nchunks, gsz, c->dgrad.as<double>());
    c->launches += 2;
    KS_CUDA(c, cudaGetLastError());
    return KS_OK;
}

template <int CH>
int launch_adjoint_mixed_ch(ks_context* c, int ntot, const double* dt, const double* dn) {
    if (ntot > 32 * kMaxSplatWords) return fail(c, KS_ERR_ARGUMENT, "the mixed adjoint takes at most %d splats (%d)", 32 * kMaxSplatWords, ntot);
    // the per-warp accumulator in shared memory while it leaves at least eight warps per SM, else the
    // unit's block of global memory
    // (384-thread blocks cap the element phase at 170 registers, with some spills, for 12 warps per SM
    // instead of 8: 6% faster at configuration 3, the same sums)
    bool global_acc = false;
    int w384 = adjoint_blocks<CH, 384>(c, ntot, false) * 12, w256 = adjoint_blocks<CH, 256>(c, ntot, false) * 8,
        w128 = adjoint_blocks<CH, 128>(c, ntot, false) * 4, w64 = adjoint_blocks<CH, 64>(c, ntot, false) * 2;
    if (std::max(std::max(w384, w256), std::max(w128, w64)) < 8) {
        global_acc = true;
        w384 = adjoint_blocks<CH, 384>(c, ntot, true) * 12; w256 = adjoint_blocks<CH, 256>(c, ntot, true) * 8;
        w128 = adjoint_blocks<CH, 128>(c, ntot, true) * 4; w64 = adjoint_blocks<CH, 64>(c, ntot, true) * 2;
    }
    const int best = std::max(std::max(w384, w256), std::max(w128, w64));
    if (best <= 0) return fail(c, KS_ERR_ARGUMENT, "too many splats for the mixed adjoint (%d)", ntot);
    if (w384 == best) return launch_adjoint_mixed_nt<CH, 384>(c, ntot, w384 / 12, dt, dn, global_acc);
    if (w256 == best) return launch_adjoint_mixed_nt<CH, 256>(c, ntot, w256 / 8, dt, dn, global_acc);
    if (w128 == best) return launch_adjoint_mixed_nt<CH, 128>(c, ntot, w128 / 4, dt, dn, global_acc);
    return launch_adjoint_mixed_nt<CH, 64>(c, ntot, w64 / 2, dt, dn, global_acc);
}

// The forward image with the state the reverse pass needs (FP64: stored samples, cutoffs, tails),
// the seeds (given, or those of chi^2), the reverse pass and the reduction into dparams.
int adjoint_run(ks_context* c, const ks_splat_set* sets, int nsets, const double* times, int nframes, const double* nus, int nfreq,
                double L, int precision, int nmax, double slab, const double* dstokes, int order, const double* data,
                const double* sigma, double sigma_s, const uint8_t* mask, double* chi2_out, double* dparams, int accumulate,
                double* image, const VisData* vd = nullptr) {
    if (!c->regenerated) return fail(c, KS_ERR_NOT_REGENERATED, "regenerate the context first");
    if (nsets < 0 || (nsets > 0 && !sets)) return fail(c, KS_ERR_ARGUMENT, "bad splat sets");
    if (nframes < 1 || nfreq < 1 || !times || !nus) return fail(c, KS_ERR_ARGUMENT, "need at least one frame and one frequency");
    const bool geo = precision == KS_MIXED_GEO64;   // the FP64 march under the mixed transport
    if (geo) precision = KS_MIXED;
    if (precision != KS_FP64 && precision != KS_MIXED) return fail(c, KS_ERR_ARGUMENT, "unknown precision %d for the adjoint", precision);
    if (order != KS_ORDER_SORTED && order != KS_ORDER_SCREEN) return fail(c, KS_ERR_ARGUMENT, "unknown order %d", order);
    if (!(std::isfinite(L) && L > 0)) return fail(c, KS_ERR_NONFINITE, "length unit must be finite and positive");
    if (!std::isfinite(slab)) return fail(c, KS_ERR_NONFINITE, "non-finite slab");
    if (!dparams) return fail(c, KS_ERR_ARGUMENT, "dparams is required");
    if (data && !sigma && !(std::isfinite(sigma_s) && sigma_s > 0))
        return fail(c, KS_ERR_ARGUMENT, "chi^2 needs sigma (an array, or a finite positive scalar)");
    KS_CUDA(c, cudaSetDevice(c->device));
    std::vector<double> ht(nframes), hnu(nfreq);
    KS_CUDA(c, cudaMemcpy(ht.data(), times, nframes * sizeof(double), cudaMemcpyDefault));
    KS_CUDA(c, cudaMemcpy(hnu.data(), nus, nfreq * sizeof(double), cudaMemcpyDefault));
    for (double v : ht) if (!std::isfinite(v)) return fail(c, KS_ERR_NONFINITE, "non-finite observation time");
    for (double v : hnu) if (!(std::isfinite(v) && v > 0)) return fail(c, KS_ERR_NONFINITE, "frequencies must be finite and positive");
    int ntot = 0;
    {
        int s = build_tables(c, sets, nsets, &ntot, true);
        if (s) return s;
    }
    const long long n = c->npix;
    const int N = c->st.N;
    const int ncombo = nframes * nfreq;
    const long long nrc = n * ncombo;
    // the times, the frequencies (the mixed forward pass), then per combination fv * nframes + ft its
    // time and frequency (the plain path)
    std::vector<double> hc(ht);
    hc.insert(hc.end(), hnu.begin(), hnu.end());
    hc.resize(size_t(nframes) + nfreq + 2 * size_t(ncombo));
    for (int fv = 0; fv < nfreq; ++fv)
        for (int ft = 0; ft < nframes; ++ft) {
            hc[nframes + nfreq + size_t(fv) * nframes + ft] = ht[ft];
            hc[nframes + nfreq + ncombo + size_t(fv) * nframes + ft] = hnu[fv];
        }
    KS_CUDA(c, c->combos.ensure(hc.size() * sizeof(double)));
    KS_CUDA(c, cudaMemcpyAsync(c->combos.p, hc.data(), hc.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    const double* dtimes = c->combos.as<double>();
    const double* dfreqs = dtimes + nframes;
    const double* dct = dfreqs + nfreq;
    const double* dcn = dct + ncombo;
    KS_CUDA(c, c->out_sorted.ensure(size_t(nrc) * 4 * sizeof(double)));
    KS_CUDA(c, c->seeds.ensure(size_t(nrc) * 4 * sizeof(double)));
    KS_CUDA(c, c->dgrad.ensure(size_t(std::max(ntot, 1)) * GR_COUNT * sizeof(double)));
    cudaEventRecord(c->ev0, c->stream);
    const bool mixed = precision == KS_MIXED;
    // 1. forward pass with the reverse pass's state
    StoredSamples S{};
    const int* kst = nullptr;
    const size_t tab_smem = size_t(ntot) * ST_COUNT * sizeof(double);
    if (mixed) {
        c->geo64 = geo;
        const size_t rows = size_t(ncombo) * N * c->npad;
        KS_CUDA(c, c->adj_state.ensure(rows * 27 * sizeof(float)));
        KS_CUDA(c, c->adj_act.ensure(rows));
        KS_CUDA(c, cudaMemsetAsync(c->adj_act.p, 0, rows, c->stream));
        c->fwd_gstate = c->adj_state.as<float>();
        c->fwd_gact = c->adj_act.as<unsigned char>();
        int s = launch_mixed(c, ntot, ht.data(), nframes, nfreq, L, nmax, slab, true);
        c->fwd_gstate = nullptr;
        c->fwd_gact = nullptr;
        if (s) return s;
    } else {
    if (tab_smem > 200 * 1024) return fail(c, KS_ERR_ARGUMENT, "too many splats for the FP64 adjoint (%d)", ntot);
    {
        int s = ensure_samples(c, &S);
        if (s) return s;
    }
    if (nmax >= 0) {
        KS_CUDA(c, c->kstop.ensure(size_t(n) * sizeof(int)));
        k_kstop<<<nblocks(n), kBlock, 0, c->stream>>>(S, n, N, c->st.rh * (1 + 1e-3), nmax, slab, c->kstop.as<int>());
        c->launches++;
        KS_CUDA(c, cudaGetLastError());
        kst = c->kstop.as<int>();
    }
    KS_CUDA(c, c->tails.ensure(size_t(ncombo) * (N + 1) * 4 * n * sizeof(double)));
    KS_CUDA(c, cudaFuncSetAttribute(k_tails, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tab_smem));
    k_tails<<<nblocks(nrc), kBlock, tab_smem, c->stream>>>(plan_view(c), c->st, n, S, kst, c->tab.as<double>(), ntot, dct, dcn, ncombo, L,
                                                          c->tails.as<double>(), c->out_sorted.as<double>());
    c->launches++;
    c->adjoint_launches++;
    KS_CUDA(c, cudaGetLastError());
    }
    // 2. seeds
    const long long nblk = (nrc + 255) / 256;
    double vis_chi2 = 0.0;
    if (vd) {
        // the visibilities of the image, chi^2 of the gained model and the adjoint transform of its
        // weights (frame_chi2_seed!): the DFT in the render's precision class (3xTF32 for the mixed path)
        if (ncombo != 1) return fail(c, KS_ERR_ARGUMENT, "visibility chi^2 takes one frame at one frequency");
        const int dprec = mixed ? KS_MIXED : KS_FP64;
        int s = dft_checks(c, vd->nuv, vd->psize, vd->scale, dprec);
        if (s) return s;
        const int64_t nuv = vd->nuv;
        const double *du, *dv, *dtap, *dg, *dvis;
        if ((s = dft_stage(c, 1, vd->u, nuv, &du)) || (s = dft_stage(c, 2, vd->v, nuv, &dv)) ||
            (s = dft_stage(c, 3, vd->tap, vd->tap ? nuv : 0, &dtap)) || (s = dft_stage(c, 6, vd->g, vd->g ? 2 * nuv : 0, &dg)) ||
            (s = dft_stage(c, 7, vd->vis, size_t(nuv) * 8, &dvis)))
            return s;
        KS_CUDA(c, c->dft_in[4].ensure(size_t(nuv) * 8 * sizeof(double) * 2 + size_t(nuv) * 4 * sizeof(double)));
        double* dV = c->dft_in[4].as<double>();
        double* dW = dV + nuv * 8;
        double* dS = dW + nuv * 8;
        KS_CUDA(c, cudaMemcpyAsync(dS, vd->sigma, size_t(nuv) * 4 * sizeof(double), cudaMemcpyDefault, c->stream));
        if ((s = dft_forward(c, c->out_sorted.as<double>(), KS_ORDER_SORTED, nuv, du, dv, dtap, vd->psize, vd->scale, dprec, dV))) return s;
        const int vblk = int((nuv * 4 + 255) / 256);
        KS_CUDA(c, c->dft_partial.ensure(size_t(vblk) * sizeof(double)));
        ksdft::k_chi2_weights<<<vblk, 256, 0, c->stream>>>(nuv, dV, dg, dvis, dS, dW, c->dft_partial.as<double>());
        c->launches++;
        KS_CUDA(c, cudaGetLastError());
        if ((s = dft_adjoint(c, dW, nuv, du, dv, dtap, vd->psize, vd->scale, dprec, c->seeds.as<double>(), KS_ORDER_SORTED, dprec != KS_FP64)))
            return s;
        std::vector<double> part(vblk);
        KS_CUDA(c, cudaMemcpyAsync(part.data(), c->dft_partial.p, vblk * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        KS_CUDA(c, cudaStreamSynchronize(c->stream));
        for (double p : part) vis_chi2 += p;   // fixed order
    } else if (data) {
        const double *dd = nullptr, *ds = nullptr;
        const uint8_t* dm = nullptr;
        KS_CUDA(c, c->dstage.ensure(size_t(nrc) * 4 * sizeof(double) * (sigma ? 2 : 1) + size_t(nrc)));
        // host data, sigma and mask share one staging buffer
        const bool hd = !is_device_ptr(data), hs = sigma && !is_device_ptr(sigma), hm = mask && !is_device_ptr(mask);
        double* st0 = c->dstage.as<double>();
        if (hd) { KS_CUDA(c, cudaMemcpyAsync(st0, data, size_t(nrc) * 4 * sizeof(double), cudaMemcpyHostToDevice, c->stream)); dd = st0; }
        else dd = data;
        if (sigma) {
            if (hs) { KS_CUDA(c, cudaMemcpyAsync(st0 + nrc * 4, sigma, size_t(nrc) * 4 * sizeof(double), cudaMemcpyHostToDevice, c->stream)); ds = st0 + nrc * 4; }
            else ds = sigma;
        }
        if (mask) {
            uint8_t* m0 = reinterpret_cast<uint8_t*>(st0 + nrc * 4 * (sigma ? 2 : 1));
            if (hm) { KS_CUDA(c, cudaMemcpyAsync(m0, mask, size_t(nrc), cudaMemcpyHostToDevice, c->stream)); dm = m0; }
            else dm = mask;
        }
        KS_CUDA(c, c->chi_part.ensure(size_t(nblk) * sizeof(double)));
        KS_CUDA(c, c->chi_val.ensure(sizeof(double)));
        k_chi2_seed<<<unsigned(nblk), 256, 0, c->stream>>>(c->out_sorted.as<double>(), c->perm.as<long long>(), n, ncombo, dd, ds, sigma_s, dm,
                                                           c->seeds.as<double>(), c->chi_part.as<double>());
        k_sum_partials<<<1, 256, 0, c->stream>>>(c->chi_part.as<double>(), nblk, c->chi_val.as<double>());
        c->launches += 2;
        KS_CUDA(c, cudaGetLastError());
    } else {
        const double* dsd = nullptr;
        {
            int s = stage_dev(c, c->dstage, dstokes, size_t(nrc) * 4, &dsd);
            if (s) return s;
        }
        k_sort_seed<<<nblocks(nrc, 256), 256, 0, c->stream>>>(dsd, c->perm.as<long long>(), n, ncombo, order == KS_ORDER_SCREEN ? 1 : 0,
                                                              c->seeds.as<double>());
        c->launches++;
        KS_CUDA(c, cudaGetLastError());
    }
    // 3. reverse pass and the deterministic reduction
    if (ntot > 0 && mixed) {
        // the reverse pass groups frequencies as the forward pass did
        const int ch = c->last_job.ch;
        int s = ch == 4 ? launch_adjoint_mixed_ch<4>(c, ntot, dtimes, dfreqs)
                        : (ch == 3 ? launch_adjoint_mixed_ch<3>(c, ntot, dtimes, dfreqs)
                                   : (ch == 2 ? launch_adjoint_mixed_ch<2>(c, ntot, dtimes, dfreqs) : launch_adjoint_mixed_ch<1>(c, ntot, dtimes, dfreqs)));
        if (s) return s;
    } else if (ntot > 0) {
        // per-ray slots in ray chunks of at most 4 GB, each reduced (in ray order) into dgrad
        const long long per_ray = (long long)GR_COUNT * ntot * ncombo * (long long)sizeof(double);
        const long long nr = std::max(1LL, std::min(n, (4LL << 30) / per_ray));
        KS_CUDA(c, c->slots.ensure(size_t(nr) * per_ray));
        KS_CUDA(c, cudaFuncSetAttribute(k_dual_plain, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tab_smem));
        for (long long j0 = 0; j0 < n; j0 += nr) {
            const long long m = std::min(nr, n - j0);
            KS_CUDA(c, cudaMemsetAsync(c->slots.p, 0, size_t(m) * per_ray, c->stream));
            k_dual_plain<<<nblocks(m * ncombo), kBlock, tab_smem, c->stream>>>(plan_view(c), c->st, n, S, kst, c->tab.as<double>(),
                                                                              c->gtab.as<double>(), ntot, dct, dcn, ncombo, L,
                                                                              c->tails.as<double>(), c->seeds.as<double>(),
                                                                              c->slots.as<double>(), j0, m);
            c->launches++;
            c->adjoint_launches++;
            KS_CUDA(c, cudaGetLastError());
            k_slot_reduce<<<unsigned(GR_COUNT * ntot), 256, 0, c->stream>>>(c->slots.as<double>(), m * ncombo, ntot, c->dgrad.as<double>(),
                                                                            j0 > 0 ? 1 : 0);
            c->launches++;
            KS_CUDA(c, cudaGetLastError());
        }
    }
    cudaEventRecord(c->ev1, c->stream);
    // 4. results
    const long long ng = (long long)ntot * GR_COUNT;
    if (ng > 0) {
        if (is_device_ptr(dparams)) {
            k_accumulate<<<nblocks(ng, 256), 256, 0, c->stream>>>(dparams, c->dgrad.as<double>(), ng, accumulate);
            c->launches++;
            KS_CUDA(c, cudaGetLastError());
        } else {
            std::vector<double> hg(ng);
            KS_CUDA(c, cudaMemcpyAsync(hg.data(), c->dgrad.p, ng * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
            KS_CUDA(c, cudaStreamSynchronize(c->stream));
            for (long long q = 0; q < ng; ++q) dparams[q] = (accumulate ? dparams[q] : 0.0) + hg[q];
        }
    }
    if (data && chi2_out) KS_CUDA(c, cudaMemcpyAsync(chi2_out, c->chi_val.p, sizeof(double), cudaMemcpyDefault, c->stream));
    if (vd && chi2_out) *chi2_out = vis_chi2;
    if (image) {
        int s = emit(c, c->out_sorted.as<double>(), 4, ncombo, KS_ORDER_SCREEN, image);
        if (s) return s;
    }
    KS_CUDA(c, cudaStreamSynchronize(c->stream));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    c->adjoint_ms += ms;
    if (precision != KS_FP64) return check_device_flag(c, "adjoint");
    return KS_OK;
}

}  // namespace

extern "C" {

int ks_adjoint(ks_context* c, const ks_splat_set* sets, int32_t nsets, const double* times, int32_t nframes, const double* nus,
               int32_t nfreq, double L, int32_t precision, int32_t nmax, double slab, const double* dstokes, int32_t order,
               double* dparams, int32_t accumulate) {
    if (!c || !dstokes) return KS_ERR_ARGUMENT;
    return adjoint_run(c, sets, nsets, times, nframes, nus, nfreq, L, precision, nmax, slab, dstokes, order, nullptr, nullptr, 0.0,
                       nullptr, nullptr, dparams, accumulate, nullptr);
}

int ks_chi2_gradient(ks_context* c, const ks_splat_set* sets, int32_t nsets, const double* times, int32_t nframes, const double* nus,
                     int32_t nfreq, double L, int32_t precision, int32_t nmax, double slab, const double* data, const double* sigma,
                     double sigma_scalar, const uint8_t* mask, double* chi2, double* dparams, int32_t accumulate, double* image) {
    if (!c || !data) return KS_ERR_ARGUMENT;
    return adjoint_run(c, sets, nsets, times, nframes, nus, nfreq, L, precision, nmax, slab, nullptr, KS_ORDER_SCREEN, data, sigma,
                       sigma_scalar, mask, chi2, dparams, accumulate, image);
}

// One mixed chi^2 + gradient evaluation of device-resident thermal sets against device-resident
// image-domain data, recorded into a CUDA graph: the splat and gradient tables from the parameters,
// the sample stream, the forward pass with the reverse pass's state, chi^2 and its seeds, the reverse
// pass, the fixed-order reduction into dparams, chi^2 into `chi2`. It runs one ordinary evaluation
// first (validation, buffers, launch shapes), which writes chi2 and dparams as ks_chi2_gradient does.
int ks_chi2_gradient_graph_capture(ks_context* c, const ks_splat_set* sets, int32_t nsets, const double* times, int32_t nframes,
                                   const double* nus, int32_t nfreq, double L, int32_t nmax, double slab, const double* data,
                                   const double* sigma, double sigma_scalar, const uint8_t* mask, double* chi2, double* dparams,
                                   int32_t accumulate) {
    if (!c || !sets || nsets < 1 || !data || !chi2 || !dparams) return KS_ERR_ARGUMENT;
    if (!is_device_ptr(data) || (sigma && !is_device_ptr(sigma)) || (mask && !is_device_ptr(mask)) || !is_device_ptr(chi2) ||
        !is_device_ptr(dparams))
        return fail(c, KS_ERR_ARGUMENT, "a captured chi^2 + gradient reads and writes device memory only (data, sigma, mask, chi2, dparams)");
    for (int s = 0; s < nsets; ++s)
        if (sets[s].nsplat > 0 && !is_device_ptr(sets[s].params))
            return fail(c, KS_ERR_ARGUMENT, "set %d: a graph reads device-resident parameters", s);
    release_graph(c->cgraph, c->cgraph_exec);
    const bool counting = c->count_events;
    c->count_events = false;
    int status = adjoint_run(c, sets, nsets, times, nframes, nus, nfreq, L, KS_MIXED, nmax, slab, nullptr, KS_ORDER_SCREEN, data, sigma,
                             sigma_scalar, mask, chi2, dparams, accumulate, nullptr);
    c->count_events = counting;
    if (status) return status;
    int ntot = 0;
    for (int s = 0; s < nsets; ++s) ntot += sets[s].nsplat;
    const long long n = c->npix;
    const int ncombo = nframes * nfreq;
    const long long nrc = n * ncombo;
    const long long nblk = (nrc + 255) / 256;
    const size_t rows = size_t(ncombo) * c->st.N * c->npad;
    const double* dtimes = c->combos.as<double>();   // as the ordinary evaluation wrote them
    const double* dfreqs = dtimes + nframes;
    const int ch = c->last_job.ch;
    KS_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed));
    c->capturing = true;
    status = capture_tables(c, sets, nsets, ntot, true);
    if (status == KS_OK && ntot > 0) {
        // the forward pass with the reverse pass's state
        c->geo64 = false;
        if (cudaMemsetAsync(c->adj_act.p, 0, rows, c->stream) != cudaSuccess) status = fail(c, KS_ERR_DEVICE, "graph capture: activity reset");
        c->fwd_gstate = c->adj_state.as<float>();
        c->fwd_gact = c->adj_act.as<unsigned char>();
        if (status == KS_OK) status = launch_mixed(c, ntot, nullptr, nframes, nfreq, L, nmax, slab, true);
        c->fwd_gstate = nullptr;
        c->fwd_gact = nullptr;
    }
    if (status == KS_OK) {
        k_chi2_seed<<<unsigned(nblk), 256, 0, c->stream>>>(c->out_sorted.as<double>(), c->perm.as<long long>(), n, ncombo, data, sigma,
                                                           sigma_scalar, mask, c->seeds.as<double>(), c->chi_part.as<double>());
        k_sum_partials<<<1, 256, 0, c->stream>>>(c->chi_part.as<double>(), nblk, c->chi_val.as<double>());
        if (cudaGetLastError() != cudaSuccess) status = fail(c, KS_ERR_DEVICE, "graph capture: chi^2 seeds");
    }
    if (status == KS_OK && ntot > 0)
        status = ch == 4 ? launch_adjoint_mixed_ch<4>(c, ntot, dtimes, dfreqs)
                         : (ch == 3 ? launch_adjoint_mixed_ch<3>(c, ntot, dtimes, dfreqs)
                                    : (ch == 2 ? launch_adjoint_mixed_ch<2>(c, ntot, dtimes, dfreqs) : launch_adjoint_mixed_ch<1>(c, ntot, dtimes, dfreqs)));
    const long long ng = (long long)ntot * GR_COUNT;
    if (status == KS_OK && ng > 0) {
        k_accumulate<<<nblocks(ng, 256), 256, 0, c->stream>>>(dparams, c->dgrad.as<double>(), ng, accumulate);
        if (cudaGetLastError() != cudaSuccess) status = fail(c, KS_ERR_DEVICE, "graph capture: gradient");
    }
    if (status == KS_OK && cudaMemcpyAsync(chi2, c->chi_val.p, sizeof(double), cudaMemcpyDeviceToDevice, c->stream) != cudaSuccess)
        status = fail(c, KS_ERR_DEVICE, "graph capture: chi^2");
    cudaGraph_t g = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(c->stream, &g);
    c->capturing = false;
    if (status != KS_OK || ec != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return status != KS_OK ? status : fail(c, KS_ERR_DEVICE, "graph capture: %s", cudaGetErrorString(ec));
    }
    cudaGraphExec_t ex = nullptr;
    const cudaError_t ei = cudaGraphInstantiate(&ex, g, 0);
    if (ei != cudaSuccess) {
        cudaGraphDestroy(g);
        cudaGetLastError();
        return fail(c, KS_ERR_DEVICE, "graph instantiation: %s", cudaGetErrorString(ei));
    }
    c->cgraph = g;
    c->cgraph_exec = ex;
    c->cgraph_bufs = chi2_graph_buffers(c);
    return KS_OK;
}

// Replay the captured chi^2 + gradient evaluation on the context stream; with wait, synchronise and
// report a kernel whose bounded wait gave up.
int ks_chi2_gradient_graph_launch(ks_context* c, int32_t wait) {
    if (!c) return KS_ERR_ARGUMENT;
    if (!c->cgraph_exec) return fail(c, KS_ERR_ARGUMENT, "no captured chi^2 + gradient graph");
    if (chi2_graph_buffers(c) != c->cgraph_bufs)
        return fail(c, KS_ERR_ARGUMENT, "a later call reallocated buffers the graph uses: capture again");
    KS_CUDA(c, cudaGraphLaunch(c->cgraph_exec, c->stream));
    c->launches++;
    if (!wait) return KS_OK;
    KS_CUDA(c, cudaStreamSynchronize(c->stream));
    return check_device_flag(c, "chi^2 + gradient graph replay");
}

}  // extern "C"

namespace {

// J v of the image for one chunk of K directions (dirs: K x nparams, each laid out like dparams)
template <class S, int K>
int jvp_chunk(ks_context* c, int ntot, const double* dparams_dev, const double* ddirs, long long dstride, const double* dct,
              const double* dcn, int ncombo, double L, int nmax, double slab, double* img_sorted, double* out_sorted, int lnL_dir = -1) {
    KS_CUDA(c, c->jvp_tab.ensure(size_t(std::max(ntot, 1)) * ST_COUNT * sizeof(Dual<S, K>)));
    Dual<S, K>* dt = c->jvp_tab.as<Dual<S, K>>();
    if (ntot > 0) {
        k_dual_table<S, K><<<nblocks(ntot, 64), 64, 0, c->stream>>>(ntot, dparams_dev, ddirs, dstride, c->tab.as<double>(),
                                                                    c->gtab.as<double>(), dt);
        c->launches++;
        KS_CUDA(c, cudaGetLastError());
    }
    const long long nrc = c->npix * ncombo;
    if constexpr (std::is_same<S, float>::value)
        k_jvp_stream<K><<<nblocks(nrc, 64), 64, 0, c->stream>>>(plan_view(c), c->st, c->npix, dt, ntot, dct, dcn, ncombo, L, nmax, slab,
                                                                c->stream_buf.as<float>(), img_sorted, out_sorted, lnL_dir);
    else
        k_jvp<S, K><<<nblocks(nrc, 64), 64, 0, c->stream>>>(plan_view(c), c->st, c->npix, dt, ntot, dct, dcn, ncombo, L, nmax, slab, img_sorted,
                                                            out_sorted, lnL_dir);
    c->launches++;
    c->adjoint_launches++;
    KS_CUDA(c, cudaGetLastError());
    return KS_OK;
}

}  // namespace

extern "C" {

}  // extern "C"

namespace {

// ks_jvp; with lnL, one direction: d/d(ln L) (dirs ignored), exact through a dual step length
int jvp_impl(ks_context* c, const ks_splat_set* sets, int32_t nsets, const double* times, int32_t nframes, const double* nus, int32_t nfreq,
             double L, int32_t precision, int32_t nmax, double slab, const double* dirs, int32_t ndir, double* dimage, int32_t order,
             double* image, bool lnL) {
    if (!c || (!dirs && !lnL) || !dimage || ndir < 1) return KS_ERR_ARGUMENT;
    if (!c->regenerated) return fail(c, KS_ERR_NOT_REGENERATED, "regenerate the context first");
    if (nsets < 1 || !sets) return fail(c, KS_ERR_ARGUMENT, "bad splat sets");
    if (nframes < 1 || nfreq < 1 || !times || !nus) return fail(c, KS_ERR_ARGUMENT, "need at least one frame and one frequency");
    const bool geo = precision == KS_MIXED_GEO64;
    if (geo) precision = KS_MIXED;
    if (precision != KS_FP64 && precision != KS_MIXED) return fail(c, KS_ERR_ARGUMENT, "unknown precision %d for the JVP", precision);
    if (order != KS_ORDER_SORTED && order != KS_ORDER_SCREEN) return fail(c, KS_ERR_ARGUMENT, "unknown order %d", order);
    if (!(std::isfinite(L) && L > 0)) return fail(c, KS_ERR_NONFINITE, "length unit must be finite and positive");
    KS_CUDA(c, cudaSetDevice(c->device));
    std::vector<double> ht(nframes), hnu(nfreq);
    KS_CUDA(c, cudaMemcpy(ht.data(), times, nframes * sizeof(double), cudaMemcpyDefault));
    KS_CUDA(c, cudaMemcpy(hnu.data(), nus, nfreq * sizeof(double), cudaMemcpyDefault));
    for (double v : ht) if (!std::isfinite(v)) return fail(c, KS_ERR_NONFINITE, "non-finite observation time");
    for (double v : hnu) if (!(std::isfinite(v) && v > 0)) return fail(c, KS_ERR_NONFINITE, "frequencies must be finite and positive");
    int ntot = 0;
    {
        int s = build_tables(c, sets, nsets, &ntot, true);
        if (s) return s;
    }
    // the raw parameters of all sets, concatenated (21 x ntot) on the device
    const long long np = (long long)ntot * 21;
    std::vector<double> hp(np);
    {
        long long off = 0;
        for (int s = 0; s < nsets; ++s) {
            const size_t cnt = size_t(21) * sets[s].nsplat;
            if (cnt) KS_CUDA(c, cudaMemcpy(hp.data() + off, sets[s].params, cnt * sizeof(double), cudaMemcpyDefault));
            off += cnt;
        }
    }
    const int K = ndir == 1 ? 1 : 8;
    const int nchunk = (ndir + K - 1) / K;
    // directions padded to whole chunks
    std::vector<double> hd(size_t(nchunk) * K * np, 0.0);
    if (!lnL) KS_CUDA(c, cudaMemcpy(hd.data(), dirs, size_t(ndir) * np * sizeof(double), cudaMemcpyDefault));
    for (double v : hd) if (!std::isfinite(v)) return fail(c, KS_ERR_NONFINITE, "non-finite direction");
    KS_CUDA(c, c->jvp_in.ensure((hp.size() + hd.size() + 1) * sizeof(double)));
    double* dp = c->jvp_in.as<double>();
    KS_CUDA(c, cudaMemcpyAsync(dp, hp.data(), hp.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    KS_CUDA(c, cudaMemcpyAsync(dp + np, hd.data(), hd.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    const int ncombo = nframes * nfreq;
    std::vector<double> hc(2 * size_t(ncombo));
    for (int fv = 0; fv < nfreq; ++fv)
        for (int ft = 0; ft < nframes; ++ft) {
            hc[size_t(fv) * nframes + ft] = ht[ft];
            hc[ncombo + size_t(fv) * nframes + ft] = hnu[fv];
        }
    KS_CUDA(c, c->combos.ensure(hc.size() * sizeof(double)));
    KS_CUDA(c, cudaMemcpyAsync(c->combos.p, hc.data(), hc.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    const double* dct = c->combos.as<double>();
    const double* dcn = dct + ncombo;
    const long long nrc = c->npix * ncombo;
    KS_CUDA(c, c->out_sorted.ensure(size_t(nrc) * 4 * sizeof(double)));
    KS_CUDA(c, c->jvp_out.ensure(size_t(K) * nrc * 4 * sizeof(double)));
    cudaEventRecord(c->ev0, c->stream);
    if (precision == KS_MIXED) {
        // the mixed J v reads the samples of the FP32 stream (the march once for every chunk)
        c->geo64 = geo;
        int s = launch_stream(c);
        if (s) return s;
    }
    for (int ch = 0; ch < nchunk; ++ch) {
        const double* dd = dp + np + (long long)ch * K * np;
        int s;
        const int ld = lnL ? 0 : -1;
        if (precision == KS_FP64)
            s = K == 1 ? jvp_chunk<double, 1>(c, ntot, dp, dd, np, dct, dcn, ncombo, L, nmax, slab, c->out_sorted.as<double>(), c->jvp_out.as<double>(), ld)
                       : jvp_chunk<double, 8>(c, ntot, dp, dd, np, dct, dcn, ncombo, L, nmax, slab, c->out_sorted.as<double>(), c->jvp_out.as<double>(), ld);
        else
            s = K == 1 ? jvp_chunk<float, 1>(c, ntot, dp, dd, np, dct, dcn, ncombo, L, nmax, slab, c->out_sorted.as<double>(), c->jvp_out.as<double>(), ld)
                       : jvp_chunk<float, 8>(c, ntot, dp, dd, np, dct, dcn, ncombo, L, nmax, slab, c->out_sorted.as<double>(), c->jvp_out.as<double>(), ld);
        if (s) return s;
        const int nd = std::min(K, ndir - ch * K);
        s = emit(c, c->jvp_out.as<double>(), 4, int(nd * ncombo), order, dimage + (long long)ch * K * nrc * 4);
        if (s) return s;
    }
    cudaEventRecord(c->ev1, c->stream);
    if (image) {
        int s = emit(c, c->out_sorted.as<double>(), 4, ncombo, order, image);
        if (s) return s;
    }
    KS_CUDA(c, cudaStreamSynchronize(c->stream));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    c->adjoint_ms += ms;
    return KS_OK;
}

}  // namespace

extern "C" {

int ks_jvp(ks_context* c, const ks_splat_set* sets, int32_t nsets, const double* times, int32_t nframes, const double* nus, int32_t nfreq,
           double L, int32_t precision, int32_t nmax, double slab, const double* dirs, int32_t ndir, double* dimage, int32_t order,
           double* image) {
    return jvp_impl(c, sets, nsets, times, nframes, nus, nfreq, L, precision, nmax, slab, dirs, ndir, dimage, order, image, false);
}

int ks_spacetime_derivatives(ks_context* c, const ks_splat_set* sets, int32_t nsets, const double* times, int32_t nframes, const double* nus,
                             int32_t nfreq, double L, int32_t precision, int32_t nmax, double slab, double* dimage, double* image) {
    if (!c || !dimage || !sets || nsets < 1) return KS_ERR_ARGUMENT;
    if (!c->regenerated) return fail(c, KS_ERR_NOT_REGENERATED, "regenerate the context first");
    if (nframes < 1 || nfreq < 1 || !times || !nus) return fail(c, KS_ERR_ARGUMENT, "need at least one frame and one frequency");
    if (precision != KS_FP64 && precision != KS_MIXED) return fail(c, KS_ERR_ARGUMENT, "unknown precision %d", precision);
    if (!(std::isfinite(L) && L > 0)) return fail(c, KS_ERR_NONFINITE, "length unit must be finite and positive");
    KS_CUDA(c, cudaSetDevice(c->device));
    std::vector<double> ht(nframes), hnu(nfreq);
    KS_CUDA(c, cudaMemcpy(ht.data(), times, nframes * sizeof(double), cudaMemcpyDefault));
    KS_CUDA(c, cudaMemcpy(hnu.data(), nus, nfreq * sizeof(double), cudaMemcpyDefault));
    for (double v : ht) if (!std::isfinite(v)) return fail(c, KS_ERR_NONFINITE, "non-finite observation time");
    for (double v : hnu) if (!(std::isfinite(v) && v > 0)) return fail(c, KS_ERR_NONFINITE, "frequencies must be finite and positive");
    int ntot = 0;
    {
        int s = build_tables(c, sets, nsets, &ntot, false);
        if (s) return s;
    }
    const int ncombo = nframes * nfreq;
    std::vector<double> hc(2 * size_t(ncombo));
    for (int fv = 0; fv < nfreq; ++fv)
        for (int ft = 0; ft < nframes; ++ft) {
            hc[size_t(fv) * nframes + ft] = ht[ft];
            hc[ncombo + size_t(fv) * nframes + ft] = hnu[fv];
        }
    KS_CUDA(c, c->combos.ensure(hc.size() * sizeof(double)));
    KS_CUDA(c, cudaMemcpyAsync(c->combos.p, hc.data(), hc.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    const double* dct = c->combos.as<double>();
    const long long n = c->npix;
    const long long nrc = n * ncombo;
    // the dual table, the dual anchor records, then the per-(ray, combination) value + 3 partials
    const long long ntab = (long long)ntot * ST_COUNT + c->nkv;
    const size_t tab_bytes = (size_t(std::max<long long>(ntab, 1)) * sizeof(D3) + 255) / 256 * 256;
    const size_t rec_bytes = size_t(c->total_anchors) * SA_COUNT * sizeof(D3);
    KS_CUDA(c, c->jvp_tab.ensure(tab_bytes + rec_bytes));
    D3* dtab = c->jvp_tab.as<D3>();
    D3* rec = reinterpret_cast<D3*>(static_cast<unsigned char*>(c->jvp_tab.p) + tab_bytes);
    KS_CUDA(c, c->st_buf.ensure(size_t(nrc) * 16 * sizeof(double)));
    cudaEventRecord(c->ev0, c->stream);
    if (ntab > 0) {
        k_lift_table<<<nblocks(ntab, 256), 256, 0, c->stream>>>(ntab, c->tab.as<double>(), dtab);
        c->launches++;
        KS_CUDA(c, cudaGetLastError());
    }
    const PlanView P = plan_view(c);
    k_st_anchors<<<dim3(nblocks(n, 64), c->max_nanch), 64, 0, c->stream>>>(P, c->st, n, rec);
    c->launches++;
    KS_CUDA(c, cudaGetLastError());
    k_st_prefix<<<nblocks(n, 64), 64, 0, c->stream>>>(P, n, rec);
    c->launches++;
    KS_CUDA(c, cudaGetLastError());
    k_spacetime_dual<<<nblocks(nrc, 64), 64, 0, c->stream>>>(P, c->st, n, rec, dtab, ntot, dct, dct + ncombo, ncombo, L, nmax, slab,
                                                             c->st_buf.as<double>());
    c->launches++;
    c->adjoint_launches++;
    KS_CUDA(c, cudaGetLastError());
    // screen order: dimage (3 x ncombo x npix x 4) and the image
    const bool dev = is_device_ptr(dimage);
    const bool idev = image && is_device_ptr(image);
    const size_t n4 = size_t(nrc) * 4;
    KS_CUDA(c, c->stage_out.ensure(n4 * 4 * sizeof(double)));
    double* dd = dev ? dimage : c->stage_out.as<double>();
    double* di = image ? (idev ? image : c->stage_out.as<double>() + 3 * n4) : nullptr;
    k_spacetime_unpack<<<nblocks(nrc, 256), 256, 0, c->stream>>>(c->st_buf.as<double>(), c->perm.as<long long>(), n, ncombo, dd, di);
    c->launches++;
    KS_CUDA(c, cudaGetLastError());
    cudaEventRecord(c->ev1, c->stream);
    if (!dev) KS_CUDA(c, cudaMemcpyAsync(dimage, dd, n4 * 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (image && !idev) KS_CUDA(c, cudaMemcpyAsync(image, di, n4 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    KS_CUDA(c, cudaStreamSynchronize(c->stream));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    c->adjoint_ms += ms;
    return KS_OK;
}

int ks_normal_matrix(ks_context* c, const double* J, int64_t m, int64_t n, int32_t precision, double* A) {
    if (!c || !J || !A || m < 1 || n < 1) return KS_ERR_ARGUMENT;
    if (precision != KS_FP64 && precision != KS_MIXED) return fail(c, KS_ERR_ARGUMENT, "unknown precision %d", precision);
    if (n > (1 << 16)) return fail(c, KS_ERR_ARGUMENT, "too many columns (%lld)", (long long)n);
    KS_CUDA(c, cudaSetDevice(c->device));
    const double* dJ = nullptr;
    {
        int s = stage_dev(c, c->dstage, J, size_t(m) * n, &dJ);
        if (s) return s;
    }
    const bool dev = is_device_ptr(A);
    double* dA = A;
    if (!dev) { KS_CUDA(c, c->stage_out.ensure(size_t(n) * n * sizeof(double))); dA = c->stage_out.as<double>(); }
    const int nb = int((n + 31) / 32);
    if (precision == KS_FP64) {
        k_normal_fp64<<<dim3(nb, nb), dim3(32, 8), 0, c->stream>>>(m, int(n), dJ, dA);
        c->launches++;
        KS_CUDA(c, cudaGetLastError());
    } else {
        // 3xTF32 tensor-core GEMM: A = J^T J = Jt Jt^T from a split, transposed FP32 copy Jt[n][m]
        const long long ldj = ksdft::pad4(m);
        KS_CUDA(c, c->dft_a.ensure(size_t(n) * ldj * 2 * sizeof(float) + size_t(n) * n * sizeof(float)));
        float* jt_h = c->dft_a.as<float>();
        float* jt_l = jt_h + n * ldj;
        float* Af = jt_l + n * ldj;
        k_transpose_split<<<dim3(nb, unsigned((m + 31) / 32)), dim3(32, 8), 0, c->stream>>>(m, int(n), dJ, jt_h, jt_l, ldj);
        c->launches++;
        int s = gemm(c, int(n), int(n), int(m), jt_h, jt_l, ldj, jt_h, jt_l, ldj, Af, n);
        if (s) return s;
        k_to_f64<<<nblocks(n * n, 256), 256, 0, c->stream>>>(n * n, Af, dA);
        c->launches++;
        KS_CUDA(c, cudaGetLastError());
    }
    if (!dev) KS_CUDA(c, cudaMemcpyAsync(A, dA, size_t(n) * n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    KS_CUDA(c, cudaStreamSynchronize(c->stream));
    return KS_OK;
}

int ks_sample_adjoint(ks_context* c, int64_t n, const double* in, const double* Dl, const double* w, const double* R, int32_t method,
                      double* out) {
    if (!c || n < 0 || (n > 0 && (!in || !Dl || !w || !R || !out))) return KS_ERR_ARGUMENT;
    if (method != 0 && method != 1) return fail(c, KS_ERR_ARGUMENT, "method must be 0 (structured) or 1 (duals)");
    if (n == 0) return KS_OK;
    KS_CUDA(c, cudaSetDevice(c->device));
    const size_t sizes[4] = {size_t(n) * 11, size_t(n), size_t(n) * 4, size_t(n) * 4};
    const double* src[4] = {in, Dl, w, R};
    const double* dev[4];
    for (int q = 0; q < 4; ++q) {
        int s = stage_dev(c, c->dft_in[q], src[q], sizes[q], &dev[q]);
        if (s) return s;
    }
    const bool dout = is_device_ptr(out);
    double* o = out;
    if (!dout) { KS_CUDA(c, c->stage_out.ensure(size_t(n) * 31 * sizeof(double))); o = c->stage_out.as<double>(); }
    k_sample_adjoint<<<nblocks(n), kBlock, 0, c->stream>>>(n, dev[0], dev[1], dev[2], dev[3], method, o);
    c->launches++;
    KS_CUDA(c, cudaGetLastError());
    if (!dout) KS_CUDA(c, cudaMemcpyAsync(out, o, size_t(n) * 31 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    KS_CUDA(c, cudaStreamSynchronize(c->stream));
    return KS_OK;
}

int ks_vis_chi2_gradient(ks_context* c, const ks_splat_set* sets, int32_t nsets, double t_obs, double nu, double L, int32_t precision,
                         int32_t nmax, double slab, int64_t nuv, const double* u, const double* v, const double* tap, const double* g,
                         const double* vis, const double* sigma, double psize, double scale, double* chi2, double* dparams,
                         int32_t accumulate, double* image) {
    if (!c || !u || !v || !vis || !sigma || nuv < 1) return KS_ERR_ARGUMENT;
    const VisData vd{nuv, u, v, tap, g, vis, sigma, psize, scale};
    return adjoint_run(c, sets, nsets, &t_obs, 1, &nu, 1, L, precision, nmax, slab, nullptr, KS_ORDER_SCREEN, nullptr, nullptr, 0.0,
                       nullptr, chi2, dparams, accumulate, image, &vd);
}

int ks_autotune(ks_context* c, const ks_splat_set* sets, int32_t nsets, const double* times, int32_t nframes, const double* nus,
                int32_t nfreq, double L, int32_t nmax, double slab, int32_t trials, int32_t* block, int32_t* units, double* best_ms) {
    if (!c || trials < 1) return KS_ERR_ARGUMENT;
    if (!c->regenerated) return fail(c, KS_ERR_NOT_REGENERATED, "regenerate the context first");
    KS_CUDA(c, cudaSetDevice(c->device));
    const long long n4 = c->npix * (long long)nframes * nfreq * 4;
    if (nframes < 1 || nfreq < 1) return fail(c, KS_ERR_ARGUMENT, "need at least one frame and one frequency");
    KS_CUDA(c, c->st_buf.ensure(size_t(n4) * sizeof(double)));
    const int cand_nt[3] = {384, 256, 128}, cand_u[4] = {2, 4, 8, 16};
    double best = 1e300;
    int bnt = 0, bu = 0;
    const int save_nt = c->tune_nt, save_u = c->tune_units;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 4; ++b) {
            c->tune_nt = cand_nt[a]; c->tune_units = cand_u[b];
            int s = ks_render(c, sets, nsets, times, nframes, nus, nfreq, L, KS_MIXED, nmax, slab, c->st_buf.as<double>(), KS_ORDER_SORTED);
            if (s) { c->tune_nt = save_nt; c->tune_units = save_u; return s; }
            const double before = c->kernel_ms;
            for (int t = 0; t < trials; ++t) {
                s = ks_render(c, sets, nsets, times, nframes, nus, nfreq, L, KS_MIXED, nmax, slab, c->st_buf.as<double>(), KS_ORDER_SORTED);
                if (s) { c->tune_nt = save_nt; c->tune_units = save_u; return s; }
            }
            const double ms = (c->kernel_ms - before) / trials;
            if (ms < best) { best = ms; bnt = cand_nt[a]; bu = cand_u[b]; }
        }
    c->tune_nt = bnt; c->tune_units = bu;
    if (block) *block = bnt;
    if (units) *units = bu;
    if (best_ms) *best_ms = best;
    return KS_OK;
}

int ks_adjoint_stats(ks_context* c, double* adjoint_ms, long long* launches, int reset) {
    if (!c) return KS_ERR_ARGUMENT;
    if (adjoint_ms) *adjoint_ms = c->adjoint_ms;
    if (launches) *launches = c->adjoint_launches;
    if (reset) { c->adjoint_ms = 0.0; c->adjoint_launches = 0; }
    return KS_OK;
}

}  // extern "C"

// ---- visibilities (device_visibilities.jl:53-111) ------------------------------------------------

namespace {

// Stage the DFT inputs (host or device) into device buffers; returns device pointers.
int dft_stage(ks_context* c, int slot, const double* src, size_t count, const double** dev) {
    if (!src) { *dev = nullptr; return KS_OK; }
    return stage_in(c, c->dft_in[slot], src, count * sizeof(double), reinterpret_cast<const void**>(dev));
}

int dft_checks(ks_context* c, int64_t nuv, double psize, double scale, int32_t precision) {
    if (!c->regenerated) return fail(c, KS_ERR_NOT_REGENERATED, "regenerate the context first (the screen and its sort order)");
    if (nuv < 1) return fail(c, KS_ERR_ARGUMENT, "need at least one baseline");
    if (!(std::isfinite(psize) && psize > 0 && std::isfinite(scale))) return fail(c, KS_ERR_NONFINITE, "pixel size and scale must be finite");
    if (precision != KS_FP64 && precision != KS_MIXED) return fail(c, KS_ERR_ARGUMENT, "unknown precision %d", precision);
    return KS_OK;
}

// The twiddle tables of the separable transform: Tv[j][2k + c] (m_j, v_k, plain FP32, read by the
// combine and seed kernels) and the split GEMM operands Tu[i][2k + c] (the adjoint's B, K = 2 nuv) and
// TuT[2k + c][i] (the forward's B, K = na), both from (l_i, u_k).
struct Twiddles {
    float *tu_h, *tu_l, *tut_h, *tut_l;
    long long ldu, ldut;
};

Twiddles twiddle_layout(ks_context* c, int64_t nuv) {
    Twiddles t;
    const int na = c->nalpha;
    t.ldu = ksdft::pad4(2 * nuv);
    t.ldut = ksdft::pad4(na);
    t.tu_h = c->dft_tu.as<float>();
    t.tu_l = t.tu_h + na * t.ldu;
    t.tut_h = t.tu_l + na * t.ldu;
    t.tut_l = t.tut_h + 2 * nuv * t.ldut;
    return t;
}

int dft_twiddles(ks_context* c, int64_t nuv, const double* du, const double* dv, double psize) {
    const int na = c->nalpha, nb = c->nbeta;
    KS_CUDA(c, c->dft_tu.ensure((size_t(na) * ksdft::pad4(2 * nuv) * 2 + size_t(2 * nuv) * ksdft::pad4(na) * 2) * sizeof(float)));
    KS_CUDA(c, c->dft_tv.ensure(size_t(nb) * 2 * nuv * sizeof(float)));
    const Twiddles t = twiddle_layout(c, nuv);
    const long long nu = (long long)na * nuv;
    ksdft::k_twiddle_split<<<nblocks(nu, 256), 256, 0, c->stream>>>(na, -1.0, psize, nuv, du, 0, t.tu_h, t.tu_l, t.ldu);
    ksdft::k_twiddle_split<<<nblocks(nu, 256), 256, 0, c->stream>>>(na, -1.0, psize, nuv, du, 1, t.tut_h, t.tut_l, t.ldut);
    ksdft::k_twiddle<<<nblocks((long long)nb * nuv, 256), 256, 0, c->stream>>>(nb, 1.0, psize, nuv, dv, c->dft_tv.as<float>(), 2 * nuv);
    c->launches += 3;
    KS_CUDA(c, cudaGetLastError());
    return KS_OK;
}

// cuTensorMapEncodeTiled from the driver, through the runtime (no link against libcuda)
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess && q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    });
    return fn;
}

// A split operand (rows x K floats, row stride ld) as 128-row x 32-float boxes with the 128-byte
// swizzle; reads past K or past the last row are zero-filled.
bool operand_map(CUtensorMap* m, const float* p, long long rows, long long K, long long ld) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc || (reinterpret_cast<uintptr_t>(p) & 15) || (ld & 3)) return false;
    cuuint64_t dims[2] = {cuuint64_t(K), cuuint64_t(rows)};
    cuuint64_t strides[1] = {cuuint64_t(ld) * sizeof(float)};
    cuuint32_t box[2] = {cuuint32_t(ksdft::TC_BK), cuuint32_t(ksdft::TC_BM)};
    cuuint32_t estr[2] = {1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(p), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// C[M][N] = A[M][K] B[N][K]^T in 3xTF32 from split operands (ksdft): the tcgen05 kernel unless the
// context selects the mma.sync fallback. Outside a graph capture, the tcgen05 path reads the device
// flag after the launch, so a wait that gave up fails the call with KS_ERR_TIMEOUT.
int gemm(ks_context* c, int M, int N, int K, const float* Ah, const float* Al, long long lda, const float* Bh, const float* Bl, long long ldb,
         float* C, long long ldc) {
    if (M < 1 || N < 1) return KS_OK;
    if (K < 1) {
        KS_CUDA(c, cudaMemset2DAsync(C, size_t(ldc) * sizeof(float), 0, size_t(N) * sizeof(float), size_t(M), c->stream));
        return KS_OK;
    }
    c->launches++;
    c->kernel_launches++;
    const bool timed = !c->capturing;
    if (c->tensor_path == 1) {
        dim3 grid(unsigned((N + ksdft::BN - 1) / ksdft::BN), unsigned((M + ksdft::BM - 1) / ksdft::BM));
        if (timed) cudaEventRecord(c->evg0, c->stream);
        ksdft::k_gemm_3xtf32<<<grid, ksdft::NTHREADS, 0, c->stream>>>(M, N, K, Ah, Al, lda, Bh, Bl, ldb, C, ldc);
        KS_CUDA(c, cudaGetLastError());
    } else {
        CUtensorMap tah, tal, tbh, tbl;
        if (!operand_map(&tah, Ah, M, K, lda) || !operand_map(&tal, Al, M, K, lda) || !operand_map(&tbh, Bh, N, K, ldb) ||
            !operand_map(&tbl, Bl, N, K, ldb))
            return fail(c, KS_ERR_DEVICE, "tensor-core GEMM: cannot describe the operands as TMA tensor maps (M %d, N %d, K %d)", M, N, K);
        {
            static std::mutex mu;
            static unsigned long long done_devices = 0;   // one bit per device: the shared-memory opt-in is per device
            std::lock_guard<std::mutex> lock(mu);
            if (!(done_devices >> (c->device & 63) & 1)) {
                KS_CUDA(c, cudaFuncSetAttribute(ksdft::k_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, ksdft::TC_SMEM));
                done_devices |= 1ull << (c->device & 63);
            }
        }
        // a wait gives up after ~1 s at the maximum SM clock (10 ms under the staging test hook)
        const long long limit = c->stage_test ? 20000000LL : 2000000000LL;
        dim3 grid(unsigned((N + ksdft::TC_BN - 1) / ksdft::TC_BN), unsigned((M + ksdft::TC_BM - 1) / ksdft::TC_BM));
        if (timed) cudaEventRecord(c->evg0, c->stream);
        ksdft::k_gemm_tc<<<grid, ksdft::TC_THREADS, ksdft::TC_SMEM, c->stream>>>(M, N, K, tah, tal, tbh, tbl, C, ldc, limit, c->stage_test,
                                                                              c->errflag.as<unsigned>());
        KS_CUDA(c, cudaGetLastError());
    }
    if (!timed) return KS_OK;
    cudaEventRecord(c->evg1, c->stream);
    KS_CUDA(c, cudaEventSynchronize(c->evg1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->evg0, c->evg1);
    c->gemm_ms += ms;
    c->gemm_flops += 6.0 * M * double(N) * K;
    c->gemm_launches++;
    return c->tensor_path == 1 ? KS_OK : check_device_flag(c, "tensor-core GEMM");
}

// V (nuv x 4 complex) of a device image
int dft_forward(ks_context* c, const double* dimg, int32_t order, int64_t nuv, const double* du, const double* dv, const double* dtap,
                double psize, double scale, int32_t precision, double* dV) {
    const int na = c->nalpha, nb = c->nbeta;
    const long long* inv = order == KS_ORDER_SORTED ? c->inv_perm.as<long long>() : nullptr;
    if (precision == KS_FP64) {
        ksdft::k_vis_direct<<<nblocks(nuv, 64), 64, 0, c->stream>>>(na, nb, dimg, inv, nuv, du, dv, dtap, psize, scale, dV);
        c->launches++;
        c->kernel_launches++;
        KS_CUDA(c, cudaGetLastError());
        return KS_OK;
    }
    int s = dft_twiddles(c, nuv, du, dv, psize);
    if (s) return s;
    const Twiddles t = twiddle_layout(c, nuv);
    const long long lda = ksdft::pad4(na), ldt = ksdft::pad4(2 * nuv);
    KS_CUDA(c, c->dft_a.ensure(size_t(2) * 4 * nb * lda * sizeof(float)));
    KS_CUDA(c, c->dft_t.ensure(size_t(4) * nb * ldt * sizeof(float)));
    float* a_h = c->dft_a.as<float>();
    float* a_l = a_h + 4LL * nb * lda;
    ksdft::k_pack_image<<<nblocks((long long)na * nb, 256), 256, 0, c->stream>>>(dimg, inv, na, nb, a_h, a_l, lda);
    c->launches++;
    if ((s = gemm(c, 4 * nb, int(2 * nuv), na, a_h, a_l, lda, t.tut_h, t.tut_l, t.ldut, c->dft_t.as<float>(), ldt))) return s;
    ksdft::k_vis_combine<<<dim3(unsigned((nuv + ksdft::VC_K - 1) / ksdft::VC_K), 4), ksdft::VC_K * ksdft::VC_G, 0, c->stream>>>(
        nb, nuv, c->dft_t.as<float>(), ldt, c->dft_tv.as<float>(), 2 * nuv, dtap, scale, dV);
    c->launches++;
    KS_CUDA(c, cudaGetLastError());
    return KS_OK;
}

// seed (npix x 4) of device weights w (nuv x 4 complex)
int dft_adjoint(ks_context* c, const double* dw, int64_t nuv, const double* du, const double* dv, const double* dtap, double psize,
                double scale, int32_t precision, double* dseed, int32_t order, bool have_twiddles) {
    const int na = c->nalpha, nb = c->nbeta;
    const long long* inv = order == KS_ORDER_SORTED ? c->inv_perm.as<long long>() : nullptr;
    if (precision == KS_FP64) {
        ksdft::k_seed_direct<<<nblocks((long long)na * nb, 64), 64, 0, c->stream>>>(na, nb, inv, nuv, dw, du, dv, dtap, psize, scale, dseed);
        c->launches++;
        c->kernel_launches++;
        KS_CUDA(c, cudaGetLastError());
        return KS_OK;
    }
    if (!have_twiddles) {
        int s = dft_twiddles(c, nuv, du, dv, psize);
        if (s) return s;
    }
    const Twiddles t = twiddle_layout(c, nuv);
    const long long ldc = ksdft::pad4(2 * nuv);
    KS_CUDA(c, c->dft_c.ensure(size_t(2) * 4 * nb * ldc * sizeof(float)));
    const long long lds = ksdft::pad4(na);
    KS_CUDA(c, c->dft_s.ensure(size_t(4) * nb * lds * sizeof(float)));
    float* c_h = c->dft_c.as<float>();
    float* c_l = c_h + 4LL * nb * ldc;
    ksdft::k_seed_rhs<<<nblocks(nuv * 4 * nb, 256), 256, 0, c->stream>>>(nb, nuv, c->dft_tv.as<float>(), 2 * nuv, dw, dtap, scale, c_h, c_l, ldc);
    c->launches++;
    // S[(s, j)][i] = CT Tu^T: rows of the seed image, so that the unpacking reads along i
    int s = gemm(c, 4 * nb, na, int(2 * nuv), c_h, c_l, ldc, t.tu_h, t.tu_l, t.ldu, c->dft_s.as<float>(), lds);
    if (s) return s;
    ksdft::k_unpack_seed<<<nblocks((long long)na * nb, 256), 256, 0, c->stream>>>(c->dft_s.as<float>(), lds, na, nb, inv, dseed);
    c->launches++;
    KS_CUDA(c, cudaGetLastError());
    return KS_OK;
}

// copy `count` doubles from the device buffer `src` to `dst` (host or device)
int deliver(ks_context* c, const double* src, double* dst, size_t count) {
    KS_CUDA(c, cudaMemcpyAsync(dst, src, count * sizeof(double), cudaMemcpyDefault, c->stream));
    return KS_OK;
}

}  // namespace

extern "C" {

int ks_visibilities(ks_context* c, const double* image, int32_t order, int64_t nuv, const double* u, const double* v, const double* tap,
                    double psize, double scale, int32_t precision, double* V) {
    if (!c || !image || !u || !v || !V) return KS_ERR_ARGUMENT;
    int s = dft_checks(c, nuv, psize, scale, precision);
    if (s) return s;
    if (order != KS_ORDER_SORTED && order != KS_ORDER_SCREEN) return fail(c, KS_ERR_ARGUMENT, "unknown order %d", order);
    KS_CUDA(c, cudaSetDevice(c->device));
    const double *dimg, *du, *dv, *dtap;
    if ((s = dft_stage(c, 0, image, size_t(c->npix) * 4, &dimg)) || (s = dft_stage(c, 1, u, nuv, &du)) || (s = dft_stage(c, 2, v, nuv, &dv)) ||
        (s = dft_stage(c, 3, tap, tap ? nuv : 0, &dtap)))
        return s;
    KS_CUDA(c, c->dft_in[4].ensure(size_t(nuv) * 8 * sizeof(double)));
    cudaEventRecord(c->ev0, c->stream);
    if ((s = dft_forward(c, dimg, order, nuv, du, dv, dtap, psize, scale, precision, c->dft_in[4].as<double>()))) return s;
    cudaEventRecord(c->ev1, c->stream);
    if ((s = deliver(c, c->dft_in[4].as<double>(), V, size_t(nuv) * 8))) return s;
    KS_CUDA(c, cudaStreamSynchronize(c->stream));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    c->kernel_ms += ms;
    return KS_OK;
}

int ks_vis_seed(ks_context* c, const double* w, int64_t nuv, const double* u, const double* v, const double* tap, double psize, double scale,
                int32_t precision, double* seed, int32_t order) {
    if (!c || !w || !u || !v || !seed) return KS_ERR_ARGUMENT;
    int s = dft_checks(c, nuv, psize, scale, precision);
    if (s) return s;
    if (order != KS_ORDER_SORTED && order != KS_ORDER_SCREEN) return fail(c, KS_ERR_ARGUMENT, "unknown order %d", order);
    KS_CUDA(c, cudaSetDevice(c->device));
    const double *dw, *du, *dv, *dtap;
    if ((s = dft_stage(c, 0, w, size_t(nuv) * 8, &dw)) || (s = dft_stage(c, 1, u, nuv, &du)) || (s = dft_stage(c, 2, v, nuv, &dv)) ||
        (s = dft_stage(c, 3, tap, tap ? nuv : 0, &dtap)))
        return s;
    KS_CUDA(c, c->dft_in[5].ensure(size_t(c->npix) * 4 * sizeof(double)));
    if ((s = dft_adjoint(c, dw, nuv, du, dv, dtap, psize, scale, precision, c->dft_in[5].as<double>(), order, false))) return s;
    if ((s = deliver(c, c->dft_in[5].as<double>(), seed, size_t(c->npix) * 4))) return s;
    KS_CUDA(c, cudaStreamSynchronize(c->stream));
    return KS_OK;
}

int ks_frame_chi2_seed(ks_context* c, const double* image, int32_t order, int64_t nuv, const double* u, const double* v, const double* tap,
                       const double* g, const double* vis, const double* sigma, double psize, double scale, int32_t precision,
                       double* chi2, double* seed) {
    if (!c || !image || !u || !v || !vis || !sigma || !chi2 || !seed) return KS_ERR_ARGUMENT;
    int s = dft_checks(c, nuv, psize, scale, precision);
    if (s) return s;
    if (order != KS_ORDER_SORTED && order != KS_ORDER_SCREEN) return fail(c, KS_ERR_ARGUMENT, "unknown order %d", order);
    KS_CUDA(c, cudaSetDevice(c->device));
    const double *dimg, *du, *dv, *dtap, *dg, *dvis, *dsig;
    if ((s = dft_stage(c, 0, image, size_t(c->npix) * 4, &dimg)) || (s = dft_stage(c, 1, u, nuv, &du)) || (s = dft_stage(c, 2, v, nuv, &dv)) ||
        (s = dft_stage(c, 3, tap, tap ? nuv : 0, &dtap)) || (s = dft_stage(c, 6, g, g ? 2 * nuv : 0, &dg)) ||
        (s = dft_stage(c, 7, vis, size_t(nuv) * 8, &dvis)))
        return s;
    KS_CUDA(c, c->dft_in[4].ensure(size_t(nuv) * 8 * sizeof(double) * 2 + size_t(nuv) * 4 * sizeof(double)));
    double* dV = c->dft_in[4].as<double>();
    double* dW = dV + nuv * 8;
    double* dS = dW + nuv * 8;
    KS_CUDA(c, cudaMemcpyAsync(dS, sigma, size_t(nuv) * 4 * sizeof(double), cudaMemcpyDefault, c->stream));
    dsig = dS;
    KS_CUDA(c, c->dft_in[5].ensure(size_t(c->npix) * 4 * sizeof(double)));
    if ((s = dft_forward(c, dimg, order, nuv, du, dv, dtap, psize, scale, precision, dV))) return s;
    const int nblk = int((nuv * 4 + 255) / 256);
    KS_CUDA(c, c->dft_partial.ensure(size_t(nblk) * sizeof(double)));
    ksdft::k_chi2_weights<<<nblk, 256, 0, c->stream>>>(nuv, dV, dg, dvis, dsig, dW, c->dft_partial.as<double>());
    c->launches++;
    KS_CUDA(c, cudaGetLastError());
    if ((s = dft_adjoint(c, dW, nuv, du, dv, dtap, psize, scale, precision, c->dft_in[5].as<double>(), order, precision != KS_FP64))) return s;
    std::vector<double> part(nblk);
    KS_CUDA(c, cudaMemcpyAsync(part.data(), c->dft_partial.p, nblk * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if ((s = deliver(c, c->dft_in[5].as<double>(), seed, size_t(c->npix) * 4))) return s;
    KS_CUDA(c, cudaStreamSynchronize(c->stream));
    double x = 0.0;
    for (double p : part) x += p;   // fixed order: deterministic
    *chi2 = x;
    return KS_OK;
}

}  // extern "C"

// ---- the allocation-free thin image -------------------------------------------------------------

// Device address of g_noalloc_tab, looked up once per device (with that device current) by the first
// ks_thin_image_noalloc call on it. cudaGetSymbolAddress does not allocate.
static std::mutex g_noalloc_mutex;
static void* g_noalloc_addr[64] = {nullptr};

static int noalloc_table(ks_context* c, double** tab) {
    if (c->device < 0 || c->device >= 64) return fail(c, KS_ERR_DEVICE, "device index %d out of range", c->device);
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_addr[c->device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_tab);
        if (e != cudaSuccess || !p) return cuda_fail(c, e == cudaSuccess ? cudaErrorInvalidSymbol : e, "cudaGetSymbolAddress(g_noalloc_tab)");
        g_noalloc_addr[c->device] = p;
    }
    *tab = static_cast<double*>(g_noalloc_addr[c->device]);
    return KS_OK;
}

extern "C" {

int ks_thin_image_noalloc(ks_context* c, const double* params, int32_t nsplat, double t_obs, int32_t precision, double* out,
                          int32_t order) {
    if (!c) return KS_ERR_ARGUMENT;
    if (!c->regenerated) return fail(c, KS_ERR_NOT_REGENERATED, "regenerate the context first");
    if (nsplat < 0 || nsplat > kNoAllocMaxSplats)
        return fail(c, KS_ERR_ARGUMENT, "ks_thin_image_noalloc takes at most %d splats (got %d)", kNoAllocMaxSplats, nsplat);
    if (precision != KS_FP64 && precision != KS_MIXED) return fail(c, KS_ERR_ARGUMENT, "unknown precision %d", precision);
    if (order != KS_ORDER_SORTED && order != KS_ORDER_SCREEN) return fail(c, KS_ERR_ARGUMENT, "unknown order %d", order);
    if (!std::isfinite(t_obs)) return fail(c, KS_ERR_NONFINITE, "non-finite observation time");
    KS_CUDA(c, cudaSetDevice(c->device));
    if (!is_device_ptr(out) || (nsplat > 0 && !is_device_ptr(params)))
        return fail(c, KS_ERR_ARGUMENT, "ks_thin_image_noalloc needs device pointers for params and out");
    double* tab = nullptr;
    int s = noalloc_table(c, &tab);
    if (s) return s;
    const long long n = c->npix;
    if (nsplat > 0) {
        SetDesc d{KS_THIN14, 14, nsplat, 0, params, nullptr, 0.0};
        k_splat_table<<<nblocks(nsplat, 64), 64, 0, c->stream>>>(d, tab);
        c->launches++;
        KS_CUDA(c, cudaGetLastError());
    }
    const long long* perm = order == KS_ORDER_SCREEN ? c->perm.as<long long>() : nullptr;
    const size_t smem = size_t(nsplat) * ST_COUNT * (precision == KS_FP64 ? sizeof(double) : sizeof(float));
    if (precision == KS_FP64) {
        KS_CUDA(c, cudaFuncSetAttribute(k_thin<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_thin<double><<<nblocks(n), kBlock, smem, c->stream>>>(plan_view(c), c->st, n, tab, nsplat, t_obs, perm, out, nullptr, nullptr);
    } else {
        KS_CUDA(c, cudaFuncSetAttribute(k_thin<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_thin<float><<<nblocks(n), kBlock, smem, c->stream>>>(plan_view(c), c->st, n, tab, nsplat, t_obs, perm, out, nullptr, nullptr);
    }
    c->launches++;
    KS_CUDA(c, cudaGetLastError());
    KS_CUDA(c, cudaStreamSynchronize(c->stream));
    return KS_OK;
}

}  // extern "C"
