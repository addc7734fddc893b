// ks_spacetime.cuh -- the image's derivatives with respect to the spacetime block (a, theta_o, ln L)
// by forward-mode duals through the whole path, as spacetime_valgrad (src/Fit/joint.jl:74-82) takes
// them with ForwardDiff through regenerate! and the transport.
//
// Dual<double, 3> numbers (partials a, theta_o, ln L) run through the same three stages as the FP64
// path: the ray's constants from its screen point at the dual spin and inclination (build_ray: roots,
// elliptic integrals, the radial/polar/quadrature constants), the Mino step tau_total / (N + 1) and
// the Jacobi step constants; the anchors (k_st_anchors, one thread per (ray, anchor): direct Jacobi
// states, the closed-form parts and the Gauss-Legendre integrals of the smooth rates, then per-ray
// running sums); and the recurrence march between them with the polarized consumer on duals, L
// entering through the step length (k_spacetime_dual, one thread per (ray, combination)). The sorted
// order, each ray's sample count and anchor spacing, its radial turning sample and every branch follow
// the values, so the derivatives are those of the same discretised function the FP64 path computes.
#pragma once

namespace {

using namespace ks;

using D3 = Dual<double, 3>;

// One anchor of a ray (k_anchor_segments): Jacobi states at tau_m, validity, the closed-form t~/phi
// parts and the smooth integral since the previous anchor.
template <class T>
__device__ void anchor_record(const RayCT<T>& R, const MarchRay<T>& M, const SpacetimeT<T>& st, int m, int Man, T dtau, JS<T>& xr,
                              JS<T>& xt, bool& ok, T& At, T& Ap, T& St, T& Sp) {
    const int k = 1 + m * Man;
    const T tau = double(k) * dtau;
    xr = xr_at(R, tau);
    xt = xt_at(R, tau);
    T th, cth;
    bool nu;
    polar_cos(M, xt, th, cth, nu);
    ok = (tau <= R.tau_valid) && visible(M, cth);
    At = T(0.0); Ap = T(0.0); St = T(0.0); Sp = T(0.0);
    if (!(tau <= R.tau_valid)) return;
    Point<T> p = ray_point(M, xr, xt, tau);
    const T r = p.r;
    const T F = r + 2.0 * log(r);
    const T Lr = (R.scattering && tau > R.fo) ? F - 2.0 * (R.r4 + 2.0 * log(R.r4)) : -F;
    const T lp = log((r - st.rp) / r) / R.sp;
    const T lm = log((r - st.rmn) / r) / R.sm;
    const JS<T> x0 = xt_at(R, T(0.0));
    const T sn0 = x0.sn / (R.pscale * x0.dn), cn0 = x0.cn / x0.dn;
    At = Lr + R.Qt * lp + R.Qtm * lm;
    Ap = R.Qphi * lp + R.Qphim * lm + polar_closed(M, tau, p.sn, p.cn) - polar_closed(M, T(0.0), sn0, cn0);
    const T ta = (m == 0) ? T(0.0) : double(1 + (m - 1) * Man) * dtau;
    const int nsamp = (m == 0) ? 1 : Man;
    const int np = (m == 0) ? 1 : (nsamp + kAnchorPanelSamples - 1) / kAnchorPanelSamples;
    const T hp = (tau - ta) / double(np);
    for (int q = 0; q < np; ++q) {
        const T a0 = ta + double(q) * hp, b0 = (q == np - 1) ? tau : ta + double(q + 1) * hp;
        T t1, p1;
        if (R.scattering && a0 < R.fo && R.fo < b0) {
            gl_panel(R, M, a0, R.fo, t1, p1); St += t1; Sp += p1;
            gl_panel(R, M, R.fo, b0, t1, p1); St += t1; Sp += p1;
        } else {
            gl_panel(R, M, a0, b0, t1, p1); St += t1; Sp += p1;
        }
    }
}

// one dual anchor record: Jacobi states, validity, t~ and phi at the anchor (closed form + running
// smooth integral), the smooth integral since the previous anchor
enum { SA_XR = 0, SA_XT = 3, SA_OK = 6, SA_T = 7, SA_PHI = 8, SA_SEG_T = 9, SA_SEG_PHI = 10, SA_COUNT = 11 };

// The dual spacetime, ray constants and march constants of sorted ray j, with the sample count,
// anchor spacing and turning sample of the plan (the values').
__device__ void dual_ray(const PlanView& P, const Spacetime& st, long long j, SpacetimeT<D3>& sd, RayCT<D3>& RC, MarchRay<D3>& R) {
    sd.a = D3::seed(st.a, 0);
    sd.thetao = D3::seed(st.thetao, 1);
    const D3 temp = sqrt(1.0 - sd.a * sd.a);
    sd.rp = 1.0 + temp; sd.rmn = 1.0 - temp; sd.rh = sd.rp;
    const D3 co = cos(sd.thetao);
    sd.abscos = fabs(co); sd.cos2 = co * co;
    sd.N = st.N; sd.M = st.M; sd.density = st.density; sd.nmin = st.nmin;
    RC = build_ray(sd, D3(P.get(PF_ALPHA, j)), D3(P.get(PF_BETA, j)));
    const int Nj = int(P.get(PF_NSAMP, j));
    const D3 dtau = RC.tau_total / double(Nj + 1);
    R = march_ray_of(RC, sd, dtau);
    const D3 h = dtau / 2.0;
    R.dr = jstep_constants(-RC.c * h, RC.k);
    R.dth = jstep_constants(RC.pscale * h / RC.tempfac, RC.pmu);
    R.turn_k = int(P.get(PF_TURN_K, j));
    R.Manchor = int(P.get(PF_MANCHOR, j));
    R.nanch = int(P.get(PF_NANCH, j));
    R.nsamp = Nj;
    R.anchor_off = P.anchor_off[j];
}

// k_anchor_segments on duals: one thread per (sorted ray, anchor)
__global__ void __launch_bounds__(64) k_st_anchors(PlanView P, Spacetime st, long long npix, D3* __restrict__ rec) {
    const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int m = blockIdx.y;
    if (j >= npix) return;
    if (m >= int(P.get(PF_NANCH, j))) return;
    SpacetimeT<D3> sd;
    RayCT<D3> RC;
    MarchRay<D3> R;
    dual_ray(P, st, j, sd, RC, R);
    JS<D3> xr, xt;
    bool ok;
    D3 At, Ap, St, Sp;
    anchor_record(RC, R, sd, m, R.Manchor, R.dtau, xr, xt, ok, At, Ap, St, Sp);
    D3* A = rec + (R.anchor_off + m) * SA_COUNT;
    A[SA_XR] = xr.sn; A[SA_XR + 1] = xr.cn; A[SA_XR + 2] = xr.dn;
    A[SA_XT] = xt.sn; A[SA_XT + 1] = xt.cn; A[SA_XT + 2] = xt.dn;
    A[SA_OK] = D3(ok ? 1.0 : 0.0);
    A[SA_T] = At; A[SA_PHI] = Ap; A[SA_SEG_T] = St; A[SA_SEG_PHI] = Sp;
}

// k_anchor_prefix on duals: t~ and phi at each anchor gain the running smooth integral
__global__ void k_st_prefix(PlanView P, long long npix, D3* __restrict__ rec) {
    const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= npix) return;
    const int nanch = int(P.get(PF_NANCH, j));
    D3 st(0.0), sp(0.0);
    for (int m = 0; m < nanch; ++m) {
        D3* A = rec + (P.anchor_off[j] + m) * SA_COUNT;
        st += A[SA_SEG_T]; sp += A[SA_SEG_PHI];
        A[SA_T] += st; A[SA_PHI] += sp;
    }
}

// The march of one ray on duals (march(), quadrature.jl:231-296), reset to the dual anchors.
template <class F>
__device__ void march_dual(const RayCT<D3>& RC, const MarchRay<D3>& R, const D3* __restrict__ rec, F& f) {
    const int N = R.nsamp;
    const D3 dtau = R.dtau;
    const D3 h = dtau / 2.0;
    const D3* A0 = rec + R.anchor_off * SA_COUNT;
    JS<D3> xr{A0[SA_XR], A0[SA_XR + 1], A0[SA_XR + 2]}, xt{A0[SA_XT], A0[SA_XT + 1], A0[SA_XT + 2]};
    Point<D3> pa = ray_point(R, xr, xt, dtau);
    D3 pca = polar_closed(R, dtau, pa.sn, pa.cn);
    D3 t = A0[SA_T], phi = A0[SA_PHI];
    {
        Sample<D3> s{t, pa.r, pa.theta, pa.cth, phi, pa.nur, pa.nuth, (dtau <= R.tau_valid) && visible(R, pa.cth)};
        f(1, s);
    }
    int next_anchor = 1 + R.Manchor;
    int m = 1;
    for (int k = 2; k <= N; ++k) {
        const D3 ta = double(k - 1) * dtau, tb = double(k) * dtau;
        xr = jstep(xr, R.dr, R.k);
        xt = jstep(xt, R.dth, R.pmu);
        Point<D3> pm = ray_point(R, xr, xt, ta + h);
        const bool anchor = (k == next_anchor);
        const D3* Am = rec + (R.anchor_off + m) * SA_COUNT;
        if (anchor) {
            xr = JS<D3>{Am[SA_XR], Am[SA_XR + 1], Am[SA_XR + 2]};
            xt = JS<D3>{Am[SA_XT], Am[SA_XT + 1], Am[SA_XT + 2]};
        } else {
            xr = jstep(xr, R.dr, R.k);
            xt = jstep(xt, R.dth, R.pmu);
        }
        Point<D3> pb = ray_point(R, xr, xt, tb);
        D3 pcb = polar_closed(R, tb, pb.sn, pb.cn);
        if (k == R.turn_k) {
            const D3 fo = R.fo_d;
            const JS<D3> p1r = xr_at(RC, (ta + fo) / 2.0), p1t = xt_at(RC, (ta + fo) / 2.0);
            const JS<D3> p2r = xr_at(RC, (fo + tb) / 2.0), p2t = xt_at(RC, (fo + tb) / 2.0);
            const JS<D3> ptt = xt_at(RC, fo);
            Point<D3> pt = turning_point(R, ptt);
            Point<D3> p1 = ray_point(R, p1r, p1t, (ta + fo) / 2.0);
            Point<D3> p2 = ray_point(R, p2r, p2t, (fo + tb) / 2.0);
            D3 pct = polar_closed(R, fo, pt.sn, pt.cn);
            D3 It1, Ip1, It2, Ip2;
            increment(R, pa, p1, pt, ta, fo, pca, pct, It1, Ip1);
            increment(R, pt, p2, pb, fo, tb, pct, pcb, It2, Ip2);
            t += It1 + It2; phi += Ip1 + Ip2;
        } else {
            D3 It, Ip;
            increment(R, pa, pm, pb, ta, tb, pca, pcb, It, Ip);
            t += It; phi += Ip;
        }
        if (anchor) {
            if (Am[SA_OK].v != 0.0) { t = Am[SA_T]; phi = Am[SA_PHI]; }
            ++m;
            next_anchor += R.Manchor;
        }
        Sample<D3> s{t, pb.r, pb.theta, pb.cth, phi, pb.nur, pb.nuth, (tb <= R.tau_valid) && visible(R, pb.cth)};
        f(k, s);
        pa = pb;
        pca = pcb;
    }
}

// RadiativeTransport (transport.jl:171-198, polarized.jl:121-150, populations.jl:70-104) on dual
// samples: the splat table and knots have zero partials, the sample position, its emission time,
// the local frame (spin, constants of motion), the step length (spin, Mino step, L) carry them.
struct SpacetimeSink {
    const D3* tab; int ntot;
    const D3* knots;
    double t_obs, nu, alpha, beta, rh_lo, slab;
    D3 Lnu, a, dtau, eta, lam, a_sin_tho;
    int nmax;
    D3 P[16], S[4];
    double zprev; int wn; bool inside, crossed, zset;

    __device__ void init() {
        for (int q = 0; q < 16; ++q) P[q] = D3((q % 5 == 0) ? 1.0 : 0.0);
        for (int q = 0; q < 4; ++q) S[q] = D3(0.0);
        wn = 0; inside = false; crossed = false; zset = false; zprev = 0.0;
    }
    __device__ void wind(double z) {   // step.jl:379-398
        if (!zset) { zprev = z; zset = true; inside = fabs(z) < slab; crossed = false; return; }
        bool inside_now = fabs(z) < slab;
        bool crossing = zprev * z < 0.0;
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
    __device__ void operator()(int, const Sample<D3>& s) {
        if (!(s.ok && s.r.v > rh_lo)) return;
        if (nmax >= 0) {
            wind(s.r.v * cos(s.theta.v));
            if (wn > nmax) return;
        }
        D3 x, y, z, sth, cth;
        ks_coords(a, s.r, s.theta, s.phi, x, y, z, sth, cth);
        const D3 t = t_obs - s.t;
        D3 in[11];
        for (int q = 0; q < 11; ++q) in[q] = D3(0.0);
        bool active = false, have_frame = false;
        SampleFrame<D3> F;
        for (int i = 0; i < ntot; ++i) {
            const D3* p = tab + (long long)i * ST_COUNT;
            D3 q;
            if (!any_exponent(p, knots, t, x, y, z, q)) continue;
            const D3 G = exp(-q);
            if (!(G > kWEIGHT_CUTOFF)) continue;
            if (!have_frame) { F = sample_frame(a, s.r, s.theta, sth, cth, eta, lam, s.nur, s.nutheta); have_frame = true; }
            const LFrame<D3> lf = local_frame(F, p[ST_U1], p[ST_U2], p[ST_U3], p[ST_BHX], p[ST_BHY], p[ST_BHZ], p[ST_BZERO].v != 0.0,
                                              D3(alpha), D3(beta), a_sin_tho);
            const D3 nuf = nu / lf.g;
            const D3 thb = safe_acos(lf.cosB);
            const D3 sbv = sin(thb), cbv = cos(thb);
            const D3 ne = p[ST_NE] * G;
            const int kind = int(p[ST_KIND].v);
            Coef<D3> cf;
            if (kind == KS_POWERLAW22)
                cf = powerlaw_cs(ne, p[ST_P], p[ST_GMIN], p[ST_GSPAN], p[ST_GAMJ], p[ST_GAMA], p[ST_BMAG], nuf, sbv, cbv);
            else if (kind == KS_KAPPA22)
                cf = kappa_cs(ne, p[ST_KAP], p[ST_W], p[ST_HYP], p[ST_G43], p[ST_G2], p[ST_GQ], p[ST_GP], p[ST_GK2], p[ST_KB], p[ST_BMAG], nuf,
                              sbv, cbv);
            else
                cf = thermal_cs(ne, p[ST_TE], p[ST_F0], p[ST_KR], p[ST_BMAG], nuf, sbv, cbv);
            if (!(cf.jI > 0.0 || cf.aI > 0.0 || cf.rQ.v != 0.0 || cf.rV.v != 0.0)) continue;
            const D3 fe = cap_factor(cf.jI, cf.jQ, cf.jV, D3(0.99));
            const D3 fa = cap_factor(cf.aI, cf.aQ, cf.aV, D3(0.99));
            const D3 nh = nuf / kNU0;
            const D3 i2 = 1.0 / (nh * nh);
            const D3 jQ = cf.jQ * fe * i2, aQ = cf.aQ * fa * nh, rQ = cf.rQ * nh;
            in[0] += cf.jI * i2; in[1] += jQ * lf.c2c; in[2] += jQ * lf.s2c; in[3] += cf.jV * fe * i2;
            in[4] += nh * cf.aI; in[5] += aQ * lf.c2c; in[6] += aQ * lf.s2c; in[7] += cf.aV * fa * nh;
            in[8] += rQ * lf.c2c; in[9] += rQ * lf.s2c; in[10] += nh * cf.rV;
            active = true;
        }
        if (!active) return;
        const D3 ct = cos(s.theta);
        const D3 Dl = Lnu * (s.r * s.r + a * a * ct * ct) * dtau;
        D3 O[16], E[4];
        transfer_step(c_moments, in, in + 4, in + 8, Dl, O, E);
        D3 Pn[16];
        for (int rr = 0; rr < 4; ++rr) {
            S[rr] += P[4 * rr] * E[0] + P[4 * rr + 1] * E[1] + P[4 * rr + 2] * E[2] + P[4 * rr + 3] * E[3];
            for (int q = 0; q < 4; ++q)
                Pn[4 * rr + q] = P[4 * rr] * O[q] + P[4 * rr + 1] * O[4 + q] + P[4 * rr + 2] * O[8 + q] + P[4 * rr + 3] * O[12 + q];
        }
        for (int q = 0; q < 16; ++q) P[q] = Pn[q];
    }
};

// the splat table (and knot array) lifted to duals with zero partials
__global__ void k_lift_table(long long n, const double* __restrict__ tab, D3* __restrict__ out) {
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q < n) out[q] = D3(tab[q]);
}

// One thread per (sorted ray, combination): out[((c npix + j) 4 + s) 4 + q] = the observed Stokes s
// (q = 0) and its derivatives along a (1), theta_o (2), ln L (3).
__global__ void __launch_bounds__(64) k_spacetime_dual(PlanView P, Spacetime st, long long npix, const D3* __restrict__ rec,
                                                       const D3* __restrict__ tab, int ntot, const double* __restrict__ ct,
                                                       const double* __restrict__ cnu, int ncombo, double L, int nmax, double slab,
                                                       double* __restrict__ out) {
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= npix * ncombo) return;
    const long long j = idx % npix;
    const int c = int(idx / npix);
    SpacetimeT<D3> sd;
    RayCT<D3> RC;
    MarchRay<D3> R;
    dual_ray(P, st, j, sd, RC, R);
    SpacetimeSink sink;
    sink.tab = tab; sink.ntot = ntot; sink.knots = tab + (long long)ntot * ST_COUNT;
    const double nh = cnu[c] / kNU0;
    sink.t_obs = ct[c]; sink.nu = cnu[c];
    sink.Lnu = D3(L / nh);
    sink.Lnu.d[2] = L / nh;   // d/d(ln L)
    sink.a = sd.a; sink.rh_lo = st.rh * (1 + 1e-3); sink.dtau = R.dtau;
    sink.alpha = P.get(PF_ALPHA, j); sink.beta = P.get(PF_BETA, j); sink.eta = RC.eta; sink.lam = RC.lam;
    sink.a_sin_tho = sd.a * sin(sd.thetao); sink.slab = slab; sink.nmax = nmax;
    sink.init();
    march_dual(RC, R, rec, sink);
    const double n3 = nh * nh * nh;
    double* o = out + idx * 16;
    for (int s = 0; s < 4; ++s) {
        o[4 * s] = sink.S[s].v * n3;
        for (int q = 0; q < 3; ++q) o[4 * s + 1 + q] = sink.S[s].d[q] * n3;
    }
}

// out (sorted, value + 3 partials per Stokes) -> dimage (3 x ncombo x npix x 4) and image (ncombo x npix x 4),
// screen order through the permutation
__global__ void k_spacetime_unpack(const double* __restrict__ src, const long long* __restrict__ perm, long long npix, int ncombo,
                                   double* __restrict__ dimage, double* __restrict__ image) {
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= npix * ncombo) return;
    const long long j = idx % npix, c = idx / npix;
    const long long scr = c * npix + perm[j];
    const double* o = src + idx * 16;
    for (int s = 0; s < 4; ++s) {
        if (image) image[scr * 4 + s] = o[4 * s];
        for (int q = 0; q < 3; ++q) dimage[((long long)q * ncombo * npix + scr) * 4 + s] = o[4 * s + 1 + q];
    }
}

}  // namespace
