// ks_adjoint.cuh -- the adjoint of the polarized transport with respect to the splat parameters
// (the reference's dual sweep, src/Splats/dual_gradient.jl, for PolarizedSplats).
//
// Along a ray the observed invariant Stokes vector is the tail T_1 of T_k = E_k + O_k T_{k+1}
// (T_{N+1} = 0); for l = w_1 . T_1 the adjoint in front of sample k is w_k = O_{k-1}^T ... O_1^T w_1
// and the sample's step enters l through w_k^T (O_k T_{k+1} + Ej_k j_k). So
//   j-bar = Ej^T w exactly (E is linear in j), and (alpha-bar, rho-bar) are the partials of
//   w^T (O T + Ej j) by seven forward-mode duals through the step operator (sample_adjoint,
//   transport.jl:221-245);
//   each splat's coefficients c_i enter through c-bar . c_i: the fluid rows (logTe, logB, thB, phB,
//   u1, u2, u3) by seven duals through the frame and the thermal fits, ln n_e as c-bar . c_i itself
//   (every coefficient is proportional to the density), and the thirteen geometric rows (centre,
//   log-widths, quaternion, t0, logw, omega) as c-bar . c_i times the partials of ln G, here in
//   closed form (element_adjoint!, dual_gradient.jl:43-76).
// Samples that the forward pass skips (invalid, inside r_h (1 + 1e-3), beyond the half-orbit cutoff,
// or with no active element) have O = 1, E = 0 and no adjoint; culled splats and weights below the
// cutoff contribute nothing, as in the reference.
//
// FP64 plain path (the reference's structure, one thread per (ray, frame x frequency)):
//   k_kstop (winding_cutoff_kernel!, dual_gradient.jl:81-97) -> k_tails (polarized_tails_kernel!,
//   129-147; writes the image) -> k_dual_plain (polarized_dual_kernel!, 151-178; per-ray gradient
//   slots) -> k_slot_reduce (the deterministic sum over rays, 239-241).
#pragma once
#include "ks_transfer.cuh"

namespace ks {

// ---- per-splat constants of the gradient (FP64) ------------------------------------------------
enum GradTab { GT_DF0, GT_DKR, GT_DBT0, GT_DBT1, GT_DBT2, GT_DBP0, GT_DBP1, GT_DBP2, GT_QW, GT_QX, GT_QY, GT_QZ, GT_QN, GT_COUNT };

// gradient rows of a THERMAL21 column (polarized.jl:17-19, 0-based)
enum GradRow { GR_X, GR_Y, GR_Z, GR_S1, GR_S2, GR_S3, GR_Q1, GR_Q2, GR_Q3, GR_Q4, GR_T0, GR_LOGW, GR_LOGNE, GR_LOGTE, GR_LOGB,
               GR_THB, GR_PHB, GR_U1, GR_U2, GR_U3, GR_OMEGA, GR_COUNT };

// ---- the step adjoint (sample_adjoint, transport.jl:221-245) -------------------------------------
// in: j (4), alpha (4), rho (3) of the sample summed over elements, Dl the step length; w the adjoint
// in front of the sample, R the tail behind it. out: O (for w <- O^T w), E = Ej j, and c-bar =
// (j-bar 4, alpha-bar 4, rho-bar 3).
template <class T>
__device__ __forceinline__ void sample_adjoint(const MomentCoeffs& MC, const T* in, T Dl, const T w[4], const T R[4], T O[16], T E[4],
                                               T cb[11]) {
    using D = Dual<T, 7>;
    D al[4], rh[3];
#pragma unroll
    for (int q = 0; q < 4; ++q) al[q] = D::seed(in[4 + q], q);
#pragma unroll
    for (int q = 0; q < 3; ++q) rh[q] = D::seed(in[8 + q], 4 + q);
    D Od[16], Ejd[16];
    step_operator(MC, al, rh, D(Dl), Od, Ejd);
    D qd(T(0));
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        D row = Od[4 * r] * R[0] + Od[4 * r + 1] * R[1] + Od[4 * r + 2] * R[2] + Od[4 * r + 3] * R[3] +
                Ejd[4 * r] * in[0] + Ejd[4 * r + 1] * in[1] + Ejd[4 * r + 2] * in[2] + Ejd[4 * r + 3] * in[3];
        qd += row * w[r];
    }
#pragma unroll
    for (int q = 0; q < 16; ++q) O[q] = Od[q].v;
#pragma unroll
    for (int r = 0; r < 4; ++r) E[r] = Ejd[4 * r].v * in[0] + Ejd[4 * r + 1].v * in[1] + Ejd[4 * r + 2].v * in[2] + Ejd[4 * r + 3].v * in[3];
#pragma unroll
    for (int c = 0; c < 4; ++c) cb[c] = Ejd[c].v * w[0] + Ejd[4 + c].v * w[1] + Ejd[8 + c].v * w[2] + Ejd[12 + c].v * w[3];
#pragma unroll
    for (int q = 0; q < 7; ++q) cb[4 + q] = qd.d[q];
}

// ---- the step adjoint in structured form (the mixed path) -----------------------------------------
// In every branch of the step operator O = sum_n o_n K^n and Ej = s sum_n e_n K^n (n = 0..3), with K
// the rescaled matrix K' of step_operator (without alpha_I) and scalar coefficients that depend on
// alpha, rho only through the invariants a = aI D, a2 = |alpha_QUV|^2, r2 = |rho|^2, ar = alpha.rho
// (step.jl:64-124). So q = w^T (O R + Ej j) has
//   dq/dtheta = sum_n [do_n/dtheta <w, K^n R> + o_n <w, dK^n/dtheta R>] + s (the same with e_n and j),
// the coefficient partials by four duals in (a, a2, r2, ar), and dK/dtheta a constant sparse matrix:
// <w, dK^2 v> = <w, G K v> + <K^T w, G v>, <w, dK^3 v> = <w, G K^2 v> + <K^T w, G K v> + <K^2T w, G v>.

// sample_adjoint (transport.jl:221-245) with the structured partials; same outputs as sample_adjoint
template <class T>
__device__ __forceinline__ void sample_adjoint_structured(const MomentCoeffs& MC, const T* in, T Dl, const T w[4], const T R[4], T O[16],
                                                          T E[4], T cb[11]) {
    const T s = pow2_below(Dl);
    const T D = Dl / s;
    const T aI = in[4] * s, aQ = in[5] * s, aU = in[6] * s, aV = in[7] * s, rQ = in[8] * s, rU = in[9] * s, rV = in[10] * s;
    using D4 = Dual<T, 4>;
    const D4 a = D4::seed(aI * D, 0), a2 = D4::seed(aQ * aQ + aU * aU + aV * aV, 1), r2 = D4::seed(rQ * rQ + rU * rU + rV * rV, 2),
             ar = D4::seed(aQ * rQ + aU * rU + aV * rV, 3);
    D4 o[4], e[4];
    step_coefficients(MC, a, a2, r2, ar, D, o, e);
    T K[16];
    K[0] = 0; K[1] = aQ; K[2] = aU; K[3] = aV; K[4] = aQ; K[5] = 0; K[6] = rV; K[7] = -rU;
    K[8] = aU; K[9] = -rV; K[10] = 0; K[11] = rQ; K[12] = aV; K[13] = rU; K[14] = -rQ; K[15] = 0;
    const T* jv = in;
    T KR[4], K2R[4], K3R[4], Kj[4], K2j[4], K3j[4], Kw[4], K2w[4];
    kmul(K, R, KR); kmul(K, KR, K2R); kmul(K, K2R, K3R);
    kmul(K, jv, Kj); kmul(K, Kj, K2j); kmul(K, K2j, K3j);
    kmul_t(K, w, Kw); kmul_t(K, Kw, K2w);
    const T P[4] = {dot4(w, R), dot4(w, KR), dot4(w, K2R), dot4(w, K3R)};
    const T J[4] = {dot4(w, jv), dot4(w, Kj), dot4(w, K2j), dot4(w, K3j)};
    // the values: O = sum o_n K^n, E = s sum e_n K^n j, j-bar = Ej^T w = s sum e_n (K^n)^T w
    {
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
                O[4 * i + jj] = ((i == jj) ? o[0].v : T(0)) + o[1].v * K[4 * i + jj] + o[2].v * K2[4 * i + jj] + o[3].v * k3;
            }
        T K3w[4];
        kmul_t(K, K2w, K3w);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            E[i] = s * (e[0].v * jv[i] + e[1].v * Kj[i] + e[2].v * K2j[i] + e[3].v * K3j[i]);
            cb[i] = s * (e[0].v * w[i] + e[1].v * Kw[i] + e[2].v * K2w[i] + e[3].v * K3w[i]);
        }
    }
    // through the invariants
    T dx[4];
#pragma unroll
    for (int x = 0; x < 4; ++x) {
        T acc = T(0);
#pragma unroll
        for (int n = 0; n < 4; ++n) acc += o[n].d[x] * P[n] + s * e[n].d[x] * J[n];
        dx[x] = acc;
    }
    T g[7];
    g[0] = dx[0] * D;                                   // aI
    g[1] = dx[1] * T(2) * aQ + dx[3] * rQ;              // aQ
    g[2] = dx[1] * T(2) * aU + dx[3] * rU;
    g[3] = dx[1] * T(2) * aV + dx[3] * rV;
    g[4] = dx[2] * T(2) * rQ + dx[3] * aQ;              // rQ
    g[5] = dx[2] * T(2) * rU + dx[3] * aU;
    g[6] = dx[2] * T(2) * rV + dx[3] * aV;
    // through the explicit K of K^1, K^2, K^3
    T f1[6], f2a[6], f2b[6], f3a[6], f3b[6], f3c[6];
    T h1[6], h2a[6], h2b[6], h3a[6], h3b[6], h3c[6];
    kgen_forms(w, R, f1); kgen_forms(w, KR, f2a); kgen_forms(Kw, R, f2b);
    kgen_forms(w, K2R, f3a); kgen_forms(Kw, KR, f3b); kgen_forms(K2w, R, f3c);
    kgen_forms(w, jv, h1); kgen_forms(w, Kj, h2a); kgen_forms(Kw, jv, h2b);
    kgen_forms(w, K2j, h3a); kgen_forms(Kw, Kj, h3b); kgen_forms(K2w, jv, h3c);
#pragma unroll
    for (int t = 0; t < 6; ++t)
        g[1 + t] += o[1].v * f1[t] + o[2].v * (f2a[t] + f2b[t]) + o[3].v * (f3a[t] + f3b[t] + f3c[t]) +
                    s * (e[1].v * h1[t] + e[2].v * (h2a[t] + h2b[t]) + e[3].v * (h3a[t] + h3b[t] + h3c[t]));
    // d/d(alpha_true) = s d/d(alpha_scaled)
#pragma unroll
    for (int t = 0; t < 7; ++t) cb[4 + t] = s * g[t];
}

// ---- one thermal splat's share of the gradient at one sample (element_adjoint!) --------------------
// p: the splat's table row (in T), gt: its gradient constants (FP64), F: the sample's frame data,
// (x, y, z) its quasi-Cartesian KS position, t = t_obs - t~ the emission time. For each of the
// first nc frequencies nu[c] whose bit is set in `act`, cb(c, q) = cb[c * cstride + q * qstride] is
// the sample's c-bar at that frequency. Adds sum_c c-bar . dc/d(row) into g[21]; returns whether the
// splat contributes (inside its support, weight above the cutoff, emitting or absorbing). The frame
// and its partials are shared by the frequencies.
template <class T, int CH>
__device__ __forceinline__ bool element_adjoint(const T* p, const double* __restrict__ gt, const SampleFrame<T>& F, T x, T y, T z, T t,
                                                T alpha, T beta, T a_sin_tho, const T* nu, int nc, unsigned act, const T* cb, int cstride,
                                                int qstride, T g[GR_COUNT]) {
    // the weight and its geometric partials (Splats.jl:58-93, polarized.jl:22-29)
    const T ph = p[ST_OMEGA] * (t - p[ST_T0]);
    T sp, cp;
    fsincos(ph, sp, cp);
    const T cx = p[ST_CX] * cp - p[ST_CY] * sp, cy = p[ST_CX] * sp + p[ST_CY] * cp;
    const T d0 = x - cx, d1 = y - cy, d2 = z - p[ST_CZ];
    if (d0 * d0 + d1 * d1 + d2 * d2 > p[ST_SUPP]) return false;   // outside_support (polarized.jl:110-120)
    const T dr[3] = {d0 * cp + d1 * sp, -d0 * sp + d1 * cp, d2};
    const T* R = p + ST_R0;   // R[3 i + j]: u_j = sum_i R[3 i + j] dr_i
    T u[3], e[3];
#pragma unroll
    for (int jj = 0; jj < 3; ++jj) u[jj] = R[jj] * dr[0] + R[3 + jj] * dr[1] + R[6 + jj] * dr[2];
    e[0] = u[0] * p[ST_ES1]; e[1] = u[1] * p[ST_ES2]; e[2] = u[2] * p[ST_ES3];
    const T tt = (t - p[ST_T0]) * p[ST_INVW];
    const T q = (e[0] * e[0] + e[1] * e[1] + e[2] * e[2] + tt * tt) / T(2);
    const T G = fexp(-q);
    if (!(G > T(kWEIGHT_CUTOFF))) return false;

    // The seven fluid rows (splat_coefficients, polarized.jl:140-150): ln Te, ln B, the field's two
    // angles, the three velocity components. The frame depends on the last five only: it is formed
    // once per pair on five duals. The fits at each frequency depend on the fluid rows through four
    // scalars (ln Te with the Bessel ratios, ln B, nu_f = nu / g, cos theta_B), so they run on four
    // duals; the frame's partials of g, cos theta_B and the 2 chi rotation carry them to the rows.
    using D5 = Dual<T, 5>;
    D5 bx(p[ST_BHX]), by(p[ST_BHY]), bz(p[ST_BHZ]);
    bx.d[0] = T(gt[GT_DBT0]); by.d[0] = T(gt[GT_DBT1]); bz.d[0] = T(gt[GT_DBT2]);
    bx.d[1] = T(gt[GT_DBP0]); by.d[1] = T(gt[GT_DBP1]); bz.d[1] = T(gt[GT_DBP2]);
    const D5 u1 = D5::seed(p[ST_U1], 2), u2 = D5::seed(p[ST_U2], 3), u3 = D5::seed(p[ST_U3], 4);
    SampleFrame<D5> Fd;
#pragma unroll
    for (int k = 0; k < 4; ++k) { Fd.pu[k] = D5(F.pu[k]); Fd.pz[k] = D5(F.pz[k]); }
    Fd.lapse_inv = D5(F.lapse_inv); Fd.om_lapse = D5(F.om_lapse); Fd.sDS = D5(F.sDS); Fd.misS = D5(F.misS); Fd.ivarpi = D5(F.ivarpi);
    Fd.r = D5(F.r); Fd.sth = D5(F.sth); Fd.cth = D5(F.cth); Fd.a = D5(F.a);
    const LFrame<D5> lf = local_frame(Fd, u1, u2, u3, bx, by, bz, p[ST_BZERO] != T(0), D5(alpha), D5(beta), D5(a_sin_tho));
    using D4 = Dual<T, 4>;
    D4 Te(p[ST_TE]), f0(p[ST_F0]), kr(p[ST_KR]), Bm(p[ST_BMAG]);
    Te.d[0] = p[ST_TE]; f0.d[0] = T(gt[GT_DF0]); kr.d[0] = T(gt[GT_DKR]);
    Bm.d[1] = p[ST_BMAG];
    // the pitch angle's sine and cosine: FP32 from its cosine directly (no angle formed), FP64 through
    // safe_acos as the reference does
    const D4 cosB = D4::seed(lf.cosB.v, 3);
    D4 sbv, cbv;
    if constexpr (is_f32<T>) pitch_sc(cosB, sbv, cbv);
    else { const D4 thb = safe_acos(cosB); sbv = sin(thb); cbv = cos(thb); }
    const T s2c = lf.s2c.v, c2c = lf.c2c.v, gv = lf.g.v;
    const D4 ne(p[ST_NE] * G);
    T sc = T(0);
    T fl[7] = {T(0), T(0), T(0), T(0), T(0), T(0), T(0)};
    bool any = false;
#pragma unroll 1
    for (int c = 0; c < CH; ++c) {
        if (c >= nc || !((act >> c) & 1u)) continue;
        const T* cbc = cb + c * cstride;
        const T nufv = nu[c] / gv;
        const D4 nuf = D4::seed(nufv, 2);
        const Coef<D4> cf = thermal_cs(ne, Te, f0, kr, Bm, nuf, sbv, cbv);
        // screen_coefficients (transport.jl:265-270)
        if (!(cf.jI > T(0) || cf.aI > T(0) || cf.rQ != T(0) || cf.rV != T(0))) continue;
        const D4 fe = cap_factor(cf.jI, cf.jQ, cf.jV, D4(T(0.99)));
        const D4 fa = cap_factor(cf.aI, cf.aQ, cf.aV, D4(T(0.99)));
        const D4 nh = nuf / T(kNU0);
        const D4 i2 = D4(T(1)) / (nh * nh);
        const D4 jQ = cf.jQ * fe * i2, aQ = cf.aQ * fa * nh, rQ = cf.rQ * nh;
        // c-bar . c = A + cos(2 chi) Bq + sin(2 chi) Cq
        const D4 A = (cf.jI * i2) * cbc[0] + (cf.jV * fe * i2) * cbc[3 * qstride] + (nh * cf.aI) * cbc[4 * qstride] +
                     (cf.aV * fa * nh) * cbc[7 * qstride] + (nh * cf.rV) * cbc[10 * qstride];
        const D4 Bq = jQ * cbc[qstride] + aQ * cbc[5 * qstride] + rQ * cbc[8 * qstride];
        const D4 Cq = jQ * cbc[2 * qstride] + aQ * cbc[6 * qstride] + rQ * cbc[9 * qstride];
        sc += A.v + c2c * Bq.v + s2c * Cq.v;
        T dq[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) dq[k] = A.d[k] + c2c * Bq.d[k] + s2c * Cq.d[k];
        fl[0] += dq[0];   // ln Te
        fl[1] += dq[1];   // ln B
        // the frame's rows through nu_f = nu / g (d nu_f = -nu_f dg / g), cos theta_B and the rotation
        const T dnuf_dg = -nufv / gv;
#pragma unroll
        for (int k = 0; k < 5; ++k)
            fl[2 + k] += dq[2] * dnuf_dg * lf.g.d[k] + dq[3] * lf.cosB.d[k] + Bq.v * lf.c2c.d[k] + Cq.v * lf.s2c.d[k];
        any = true;
    }
    if (!any) return false;

    // geometric rows: g += sc * d(ln G)/d(row) = -sc * dq/d(row)
    const T gu[3] = {e[0] * p[ST_ES1], e[1] * p[ST_ES2], e[2] * p[ST_ES3]};   // dq/du
    T gdr[3];                                                                  // dq/d(dr)
#pragma unroll
    for (int ii = 0; ii < 3; ++ii) gdr[ii] = R[3 * ii] * gu[0] + R[3 * ii + 1] * gu[1] + R[3 * ii + 2] * gu[2];
    g[GR_X] += sc * gdr[0];
    g[GR_Y] += sc * gdr[1];
    g[GR_Z] += sc * gdr[2];
    g[GR_S1] += sc * e[0] * e[0];
    g[GR_S2] += sc * e[1] * e[1];
    g[GR_S3] += sc * e[2] * e[2];
    g[GR_LOGW] += sc * tt * tt;
    // the pattern phase: dq/dph through dr = rot(-ph) x - p (xy components)
    const T dqdph = gdr[0] * (dr[1] + p[ST_CY]) - gdr[1] * (dr[0] + p[ST_CX]);
    g[GR_OMEGA] -= sc * dqdph * (t - p[ST_T0]);
    g[GR_T0] -= sc * (-dqdph * p[ST_OMEGA] - tt * p[ST_INVW]);
    // the quaternion through the rotation matrix and the normalisation
    T GM[9];
#pragma unroll
    for (int ii = 0; ii < 3; ++ii)
#pragma unroll
        for (int jj = 0; jj < 3; ++jj) GM[3 * ii + jj] = dr[ii] * gu[jj];
    const T w = T(gt[GT_QW]), qx = T(gt[GT_QX]), qy = T(gt[GT_QY]), qz = T(gt[GT_QZ]);
    T gq[4];
    gq[0] = T(2) * (-qz * GM[1] + qy * GM[2] + qz * GM[3] - qx * GM[5] - qy * GM[6] + qx * GM[7]);
    gq[1] = T(2) * (qy * GM[1] + qz * GM[2] + qy * GM[3] - T(2) * qx * GM[4] - w * GM[5] + qz * GM[6] + w * GM[7] - T(2) * qx * GM[8]);
    gq[2] = T(2) * (-T(2) * qy * GM[0] + qx * GM[1] + w * GM[2] + qx * GM[3] + qz * GM[5] - w * GM[6] + qz * GM[7] - T(2) * qy * GM[8]);
    gq[3] = T(2) * (-T(2) * qz * GM[0] - w * GM[1] + qx * GM[2] + w * GM[3] - T(2) * qz * GM[4] + qy * GM[5] + qx * GM[6] + qy * GM[7]);
    const T dotq = w * gq[0] + qx * gq[1] + qy * gq[2] + qz * gq[3];
    const T inv_n = T(1.0 / gt[GT_QN]);
    g[GR_Q1] -= sc * (gq[0] - w * dotq) * inv_n;
    g[GR_Q2] -= sc * (gq[1] - qx * dotq) * inv_n;
    g[GR_Q3] -= sc * (gq[2] - qy * dotq) * inv_n;
    g[GR_Q4] -= sc * (gq[3] - qz * dotq) * inv_n;
    // ln n_e and the fluid rows
    g[GR_LOGNE] += sc;
#pragma unroll
    for (int k = 0; k < 7; ++k) g[GR_LOGTE + k] += fl[k];
    return true;
}

// The summed screen-basis coefficients of the thermal splats at one sample and frequency
// (accumulate_elements, transport.jl:254-276); false when no element is active. Same arithmetic as
// the forward consumer.
template <class T>
__device__ __forceinline__ bool sample_coefficients(const T* tab, int ntot, const SampleFrame<T>& F, T x, T y, T z, T t, T alpha, T beta,
                                                    T a_sin_tho, T nu, T out[11]) {
#pragma unroll
    for (int q = 0; q < 11; ++q) out[q] = T(0);
    bool active = false;
    for (int i = 0; i < ntot; ++i) {
        const T* p = tab + i * ST_COUNT;
        T q;
        if (!splat_exponent(p, t, x, y, z, true, q)) continue;
        T G = exp(-q);
        if (!(G > T(kWEIGHT_CUTOFF))) continue;
        LFrame<T> lf = local_frame(F, p[ST_U1], p[ST_U2], p[ST_U3], p[ST_BHX], p[ST_BHY], p[ST_BHZ], p[ST_BZERO] != T(0), alpha, beta, a_sin_tho);
        T nuf = nu / lf.g;
        T thb = acos(fmin(T(1), fmax(T(-1), lf.cosB)));
        Coef<T> cf = thermal(p[ST_NE] * G, p[ST_TE], p[ST_F0], p[ST_KR], p[ST_BMAG], nuf, thb);
        if (!(cf.jI > T(0) || cf.aI > T(0) || cf.rQ != T(0) || cf.rV != T(0))) continue;
        T fe = cap_factor(cf.jI, cf.jQ, cf.jV, T(0.99));
        T fa = cap_factor(cf.aI, cf.aQ, cf.aV, T(0.99));
        T nh = nuf / T(kNU0);
        T i2 = T(1) / (nh * nh);
        T s2c = lf.s2c, c2c = lf.c2c;
        T jQ = cf.jQ * fe * i2, aQ = cf.aQ * fa * nh, rQ = cf.rQ * nh;
        out[0] += cf.jI * i2; out[1] += jQ * c2c; out[2] += jQ * s2c; out[3] += cf.jV * fe * i2;
        out[4] += nh * cf.aI; out[5] += aQ * c2c; out[6] += aQ * s2c; out[7] += cf.aV * fa * nh;
        out[8] += rQ * c2c; out[9] += rQ * s2c; out[10] += nh * cf.rV;
        active = true;
    }
    return active;
}

// A stored FP64 sample (the reference's GeodesicSamples, direct_march.jl:71-88), [k - 1][npix] arrays.
struct StoredSamples {
    const double *t, *r, *th, *ph;
    const unsigned char* fl;
};

// What one stored sample gives the consumer: position, emission-time offset, frame data.
struct SampleGeo {
    double x, y, z, sth, cth, ts, r, th;
    bool usable, nur, nuth;
};
__device__ __forceinline__ SampleGeo stored_geo(const StoredSamples& S, long long q, double a, double rh_lo) {
    SampleGeo g;
    const unsigned f = S.fl[q];
    g.r = S.r[q]; g.th = S.th[q]; g.ts = S.t[q];
    g.usable = (f & 1u) && g.r > rh_lo;
    g.nur = (f & 2u) != 0; g.nuth = (f & 4u) != 0;
    g.x = g.y = g.z = g.sth = g.cth = 0.0;
    if (g.usable) ks_coords(a, g.r, g.th, S.ph[q], g.x, g.y, g.z, g.sth, g.cth);
    return g;
}

}  // namespace ks

namespace {

using namespace ks;

// Per-splat constants of the gradient of THERMAL21 splats: d(K0/K2)/d(logTe), d(K1/K2)/d(logTe) at
// x = 1/Theta_e (dK0/dx = -K1, dK1/dx = -K0 - K1/x), the derivatives of the field direction by its
// angles, and the normalised quaternion with its norm.
__global__ void k_grad_table(int nsplat, int first, const double* __restrict__ params, double* __restrict__ gtab) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nsplat) return;
    const double* p = params + 21LL * i;
    double* o = gtab + (long long)(first + i) * GT_COUNT;
    const double Te = exp(p[13]);
    const double xb = 1.0 / Te;
    double k0, k1;
    besselk01(xb, k0, k1);
    const double k2 = k0 + 2.0 * k1 / xb;
    if (k2 > 0) {
        const double dk0 = -k1, dk1 = -k0 - k1 / xb;
        const double dk2 = dk0 + 2.0 * dk1 / xb - 2.0 * k1 / (xb * xb);
        const double df0dx = (dk0 * k2 - k0 * dk2) / (k2 * k2), dkrdx = (dk1 * k2 - k1 * dk2) / (k2 * k2);
        o[GT_DF0] = -xb * df0dx;   // dx/dlogTe = -x
        o[GT_DKR] = -xb * dkrdx;
    } else {
        o[GT_DF0] = 0.0; o[GT_DKR] = 0.0;
    }
    const double st = sin(p[15]), ct = cos(p[15]), sp = sin(p[16]), cp = cos(p[16]);
    o[GT_DBT0] = ct * cp; o[GT_DBT1] = ct * sp; o[GT_DBT2] = -st;
    o[GT_DBP0] = -st * sp; o[GT_DBP1] = st * cp; o[GT_DBP2] = 0.0;
    const double n = sqrt(p[6] * p[6] + p[7] * p[7] + p[8] * p[8] + p[9] * p[9]);
    o[GT_QW] = p[6] / n; o[GT_QX] = p[7] / n; o[GT_QY] = p[8] / n; o[GT_QZ] = p[9] / n; o[GT_QN] = n;
}

// winding_cutoff_kernel! (dual_gradient.jl:81-97): the first sample of each ray beyond its nmax-th
// passage through |z| < slab (N + 1 when there is none)
__global__ void k_kstop(StoredSamples S, long long npix, int N, double rh_lo, int nmax, double slab, int* __restrict__ kstop) {
    const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= npix) return;
    double zprev = 0.0;
    int wn = 0;
    bool inside = false, crossed = false, zset = false;
    int stop = N + 1;
    for (int k = 1; k <= N; ++k) {
        const long long q = (long long)(k - 1) * npix + j;
        const double r = S.r[q];
        if (!((S.fl[q] & 1u) && r > rh_lo)) continue;
        const double z = r * cos(S.th[q]);
        // WindingState (step.jl:379-398)
        if (!zset) { zprev = z; zset = true; inside = fabs(z) < slab; crossed = false; }
        else {
            const bool inside_now = fabs(z) < slab;
            const bool crossing = zprev * z < 0.0;
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
        if (wn > nmax) { stop = k; break; }
    }
    kstop[j] = stop;
}

// polarized_tails_kernel! (dual_gradient.jl:129-147), FP64: one thread per (ray, combination);
// tails[((c * (N + 1) + k) * 4 + s) * npix + j] = T_{k+1} (k = 0..N), img the observed Stokes vectors.
__global__ void __launch_bounds__(128) k_tails(PlanView P, Spacetime st, long long npix, StoredSamples S, const int* __restrict__ kstop,
                                               const double* __restrict__ tab64, int ntot, const double* __restrict__ ct,
                                               const double* __restrict__ cnu, int ncombo, double L, double* __restrict__ tails,
                                               double* __restrict__ img) {
    extern __shared__ __align__(16) unsigned char smem[];
    double* tab = reinterpret_cast<double*>(smem);
    for (int q = threadIdx.x; q < ntot * ST_COUNT; q += blockDim.x) tab[q] = tab64[q];
    __syncthreads();
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= npix * ncombo) return;
    const long long j = idx % npix;
    const int c = int(idx / npix);
    const int N = st.N;
    const double a = st.a, rh_lo = st.rh * (1 + 1e-3);
    const double nu = cnu[c], t_obs = ct[c], nh = nu / kNU0, Lnu = L / nh;
    const double alpha = P.get(PF_ALPHA, j), beta = P.get(PF_BETA, j), eta = P.get(PF_ETA, j), lam = P.get(PF_LAM, j);
    const double dtau = P.get(PF_DTAU, j), a_sin_tho = a * sin(st.thetao);
    const int stop = kstop ? kstop[j] : N + 1;
    double* tl = tails + (long long)c * (N + 1) * 4 * npix + j;
    double T4[4] = {0.0, 0.0, 0.0, 0.0};
    for (int s = 0; s < 4; ++s) tl[((long long)N * 4 + s) * npix] = 0.0;
    for (int k = N; k >= 1; --k) {
        if (k < stop) {
            const SampleGeo g = stored_geo(S, (long long)(k - 1) * npix + j, a, rh_lo);
            if (g.usable) {
                SampleFrame<double> F = sample_frame(a, g.r, g.th, g.sth, g.cth, eta, lam, g.nur, g.nuth);
                double in[11];
                if (sample_coefficients(tab, ntot, F, g.x, g.y, g.z, t_obs - g.ts, alpha, beta, a_sin_tho, nu, in)) {
                    const double Sg = g.r * g.r + a * a * cos(g.th) * cos(g.th);
                    double O[16], E[4];
                    transfer_step(c_moments, in, in + 4, in + 8, Lnu * Sg * dtau, O, E);
                    double Tn[4];
                    for (int r = 0; r < 4; ++r) Tn[r] = E[r] + O[4 * r] * T4[0] + O[4 * r + 1] * T4[1] + O[4 * r + 2] * T4[2] + O[4 * r + 3] * T4[3];
                    for (int r = 0; r < 4; ++r) T4[r] = Tn[r];
                }
            }
        }
        for (int s = 0; s < 4; ++s) tl[((long long)(k - 1) * 4 + s) * npix] = T4[s];
    }
    const double n3 = nh * nh * nh;
    for (int s = 0; s < 4; ++s) img[((long long)c * npix + j) * 4 + s] = T4[s] * n3;
}

// polarized_dual_kernel! (dual_gradient.jl:151-178), FP64: one thread per (ray, combination) of the
// ray range [j0, j0 + nr), forward over the samples; the ray's share of every splat's gradient into
// its own slots grad[(row * ntot + i) * (nr ncombo) + c * nr + (j - j0)].
__global__ void __launch_bounds__(128) k_dual_plain(PlanView P, Spacetime st, long long npix, StoredSamples S, const int* __restrict__ kstop,
                                                    const double* __restrict__ tab64, const double* __restrict__ gtab, int ntot,
                                                    const double* __restrict__ ct, const double* __restrict__ cnu, int ncombo, double L,
                                                    const double* __restrict__ tails, const double* __restrict__ dstokes,
                                                    double* __restrict__ grad, long long j0, long long nr) {
    extern __shared__ __align__(16) unsigned char smem[];
    double* tab = reinterpret_cast<double*>(smem);
    for (int q = threadIdx.x; q < ntot * ST_COUNT; q += blockDim.x) tab[q] = tab64[q];
    __syncthreads();
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= nr * ncombo) return;
    const long long j = j0 + idx % nr;
    const int c = int(idx / nr);
    const long long nrc = nr * ncombo;
    const int N = st.N;
    const double a = st.a, rh_lo = st.rh * (1 + 1e-3);
    const double nu = cnu[c], t_obs = ct[c], nh = nu / kNU0, Lnu = L / nh, n3 = nh * nh * nh;
    const double alpha = P.get(PF_ALPHA, j), beta = P.get(PF_BETA, j), eta = P.get(PF_ETA, j), lam = P.get(PF_LAM, j);
    const double dtau = P.get(PF_DTAU, j), a_sin_tho = a * sin(st.thetao);
    const int stop = kstop ? kstop[j] : N + 1;
    const double* tl = tails + (long long)c * (N + 1) * 4 * npix + j;
    double w[4];
    for (int s = 0; s < 4; ++s) w[s] = dstokes[((long long)c * npix + j) * 4 + s] * n3;
    const int kend = min(stop - 1, N);
    for (int k = 1; k <= kend; ++k) {
        const SampleGeo g = stored_geo(S, (long long)(k - 1) * npix + j, a, rh_lo);
        if (!g.usable) continue;
        SampleFrame<double> F = sample_frame(a, g.r, g.th, g.sth, g.cth, eta, lam, g.nur, g.nuth);
        const double t = t_obs - g.ts;
        double in[11];
        if (!sample_coefficients(tab, ntot, F, g.x, g.y, g.z, t, alpha, beta, a_sin_tho, nu, in)) continue;
        const double Sg = g.r * g.r + a * a * cos(g.th) * cos(g.th);
        double R[4];
        for (int s = 0; s < 4; ++s) R[s] = tl[((long long)k * 4 + s) * npix];
        double O[16], E[4], cb[11];
        sample_adjoint(c_moments, in, Lnu * Sg * dtau, w, R, O, E, cb);
        for (int i = 0; i < ntot; ++i) {
            double gi[GR_COUNT];
            for (int r = 0; r < GR_COUNT; ++r) gi[r] = 0.0;
            if (!element_adjoint<double, 1>(tab + i * ST_COUNT, gtab + (long long)i * GT_COUNT, F, g.x, g.y, g.z, t, alpha, beta, a_sin_tho,
                                            &nu, 1, 1u, cb, 0, 1, gi))
                continue;
            for (int r = 0; r < GR_COUNT; ++r) grad[((long long)r * ntot + i) * nrc + idx] += gi[r];
        }
        double wn[4];
        for (int s = 0; s < 4; ++s) wn[s] = O[s] * w[0] + O[4 + s] * w[1] + O[8 + s] * w[2] + O[12 + s] * w[3];
        for (int s = 0; s < 4; ++s) w[s] = wn[s];
    }
}

// sample_adjoint of n independent samples (FP64): method 0 the structured partials, 1 the seven duals
// through the step operator; out[31 i ..] = O (16), E (4), c-bar (11)
__global__ void k_sample_adjoint(long long n, const double* __restrict__ in, const double* __restrict__ Dl, const double* __restrict__ w,
                                 const double* __restrict__ R, int method, double* __restrict__ out) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double O[16], E[4], cb[11];
    if (method == 0) sample_adjoint_structured(c_moments, in + 11 * i, Dl[i], w + 4 * i, R + 4 * i, O, E, cb);
    else sample_adjoint(c_moments, in + 11 * i, Dl[i], w + 4 * i, R + 4 * i, O, E, cb);
    double* o = out + 31 * i;
    for (int q = 0; q < 16; ++q) o[q] = O[q];
    for (int q = 0; q < 4; ++q) o[16 + q] = E[q];
    for (int q = 0; q < 11; ++q) o[20 + q] = cb[q];
}

// The deterministic sum of the per-ray slots (one block per (row, splat), a fixed tree), into the
// column-major parameter layout dparams[i * 21 + row].
__global__ void k_slot_reduce(const double* __restrict__ grad, long long nrc, int ntot, double* __restrict__ out, int accumulate) {
    __shared__ double sh[256];
    const int ri = blockIdx.x;   // row * ntot + i
    const double* g = grad + (long long)ri * nrc;
    double s = 0.0;
    for (long long q = threadIdx.x; q < nrc; q += blockDim.x) s += g[q];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) sh[threadIdx.x] += sh[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const int row = ri / ntot, i = ri % ntot;
        double* o = out + (long long)i * GR_COUNT + row;
        *o = accumulate ? *o + sh[0] : sh[0];
    }
}

// Image-domain chi^2 and its seed (_frame_seed!, src/Fit/Fit.jl:537-577): for every sorted ray j and
// combination c, r = (image - data) / sigma with data, sigma and mask in screen order; chi^2 = sum r^2
// over unmasked pixels and Stokes, seed = 2 r / sigma (zero where masked). Per-block partial sums.
__global__ void k_chi2_seed(const double* __restrict__ img, const long long* __restrict__ perm, long long npix, int ncombo,
                            const double* __restrict__ data, const double* __restrict__ sigma, double sigma_s,
                            const unsigned char* __restrict__ mask, double* __restrict__ seed, double* __restrict__ partial) {
    __shared__ double sh[256];
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    double acc = 0.0;
    if (idx < npix * ncombo) {
        const long long j = idx % npix, c = idx / npix;
        const long long scr = c * npix + perm[j];
        const bool use = mask ? mask[scr] != 0 : true;
        for (int s = 0; s < 4; ++s) {
            double sd = 0.0;
            if (use) {
                const double sg = sigma ? sigma[scr * 4 + s] : sigma_s;
                const double r = (img[idx * 4 + s] - data[scr * 4 + s]) / sg;
                acc += r * r;
                sd = 2.0 * r / sg;
            }
            seed[idx * 4 + s] = sd;
        }
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) sh[threadIdx.x] += sh[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

// sum of n partials in a fixed order (one block)
__global__ void k_sum_partials(const double* __restrict__ partial, long long n, double* __restrict__ out) {
    __shared__ double sh[256];
    double s = 0.0;
    for (long long q = threadIdx.x; q < n; q += blockDim.x) s += partial[q];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) sh[threadIdx.x] += sh[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = sh[0];
}

// screen- or sorted-order adjoint seeds (ks_adjoint's dstokes) into sorted order
__global__ void k_sort_seed(const double* __restrict__ src, const long long* __restrict__ perm, long long npix, int ncombo, int screen,
                            double* __restrict__ dst) {
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= npix * ncombo) return;
    const long long j = idx % npix, c = idx / npix;
    const long long sidx = screen ? c * npix + perm[j] : idx;
    for (int s = 0; s < 4; ++s) dst[idx * 4 + s] = src[sidx * 4 + s];
}

}  // namespace

// ---- the mixed path: a per-segment reverse pass over the FP32 sample stream --------------------------
//
// The forward pass (k_consume with MixedJob::gstate) stores, at every active (sample, ray, frequency),
// the state P_k of the segment before the sample and the summed coefficients c_k. k_adj_bounds turns
// the segments' (P, S) into the adjoint at each segment's start, w_s = (P_0 ... P_{s-1})^T w_1, and
// the tail behind each segment's end, T_s = S_{s+1} + P_{s+1} T_{s+1}. k_adj_steps walks each work
// unit (32 rays x one segment x one frame x CH frequencies) from its last sample to its first:
// w_k = P_k^T w_s, the step adjoint (structured partials) spread over the warp, T <- E + O T, and
// c-bar stored in place of c_k. k_adj_elements then evaluates the element adjoints of the (ray,
// splat) pairs that pass the support test, 32 at a time, their 21 rows summed per splat in list
// order into the warp's accumulator (shared memory). Each unit writes its own partial sums;
// k_unit_reduce adds the units in a fixed order. Two kernels keep each one's code small.

namespace {

using namespace ks;

// s: the owner's column of the block's sample data ([field][NT]); cb: the owner's c-bar column of
// [CH][11][NT]; nu: the unit's frequencies; g: the pair's 21 rows. All four in shared memory: an
// array whose address crosses the call would live on the stack.
template <int CH, int NT>
__device__ __noinline__ void element_adjoint_ool(const float* p, const double* gt, const float* s, float t_obs, float a, float a_sin_tho,
                                                 const float* nu, int nc, unsigned act, const float* cb, float* g) {
    SampleFrame<float> F;
    F.pu[0] = s[SF_PU0 * NT]; F.pu[1] = s[SF_PU1 * NT]; F.pu[2] = s[SF_PU2 * NT]; F.pu[3] = s[SF_PU3 * NT];
    F.pz[0] = s[SF_PZ0 * NT]; F.pz[1] = s[SF_PZ1 * NT]; F.pz[2] = s[SF_PZ2 * NT]; F.pz[3] = s[SF_PZ3 * NT];
    F.lapse_inv = s[SF_LI * NT]; F.om_lapse = s[SF_OL * NT]; F.sDS = s[SF_SDS * NT]; F.misS = s[SF_MIS * NT]; F.ivarpi = s[SF_IVP * NT];
    F.r = s[SF_R * NT]; F.sth = s[SF_STH * NT]; F.cth = s[SF_CTH * NT]; F.a = a;
    float gl[GR_COUNT];
#pragma unroll
    for (int r = 0; r < GR_COUNT; ++r) gl[r] = 0.f;
    element_adjoint<float, CH>(p, gt, F, s[SF_X * NT], s[SF_Y * NT], s[SF_Z * NT], t_obs - s[SF_T * NT], s[SF_ALPHA * NT], s[SF_BETA * NT],
                               a_sin_tho, nu, nc, act, cb, 11 * NT, NT, gl);
#pragma unroll
    for (int r = 0; r < GR_COUNT; ++r) g[r] = gl[r];
}

// the adjoint at each segment's start and the tail behind its end, per (ray, combination):
// bnd[((combo nseg + s) 8 + q) npix + j], q = 0..3 w, 4..7 T
__global__ void k_adj_bounds(MixedJob job, const double* __restrict__ cnu, const float* __restrict__ seg_out, const double* __restrict__ seeds,
                             float* __restrict__ bnd) {
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long ncombo = (long long)job.nframes * job.nfreq;
    if (q >= job.npix * ncombo) return;
    const long long combo = q / job.npix, j = q % job.npix;
    const int v = int(combo / job.nframes);
    const double nh = cnu[v] / kNU0, n3 = nh * nh * nh;
    const float* base = seg_out + ((combo * job.nseg) * job.npix + j) * 20;
    float* b = bnd + (combo * job.nseg) * 8 * job.npix + j;
    double w[4];
    for (int s = 0; s < 4; ++s) w[s] = seeds[(combo * job.npix + j) * 4 + s] * n3;
    for (int sg = 0; sg < job.nseg; ++sg) {
        const float* PS = base + (long long)sg * job.npix * 20;
        for (int s = 0; s < 4; ++s) b[((long long)sg * 8 + s) * job.npix] = float(w[s]);
        double wn[4];
        for (int s = 0; s < 4; ++s) wn[s] = PS[s] * w[0] + PS[4 + s] * w[1] + PS[8 + s] * w[2] + PS[12 + s] * w[3];
        for (int s = 0; s < 4; ++s) w[s] = wn[s];
    }
    double T4[4] = {0.0, 0.0, 0.0, 0.0};
    for (int sg = job.nseg - 1; sg >= 0; --sg) {
        const float* PS = base + (long long)sg * job.npix * 20;
        for (int s = 0; s < 4; ++s) b[((long long)sg * 8 + 4 + s) * job.npix] = float(T4[s]);
        double Tn[4];
        for (int r = 0; r < 4; ++r) Tn[r] = PS[16 + r] + PS[4 * r] * T4[0] + PS[4 * r + 1] * T4[1] + PS[4 * r + 2] * T4[2] + PS[4 * r + 3] * T4[3];
        for (int r = 0; r < 4; ++r) T4[r] = Tn[r];
    }
}

// The per-lane state of the step phase (T and w per frequency) and of the element phase.
template <int CH>
struct AdjSmem {
    // step phase, per-warp shares of the block's regions: T (4) and w (4) per thread and frequency;
    // step offsets, active bits, Sigma dtau per thread, scan sums
    static constexpr int kTwBytes = 32 * CH * 8 * 4;
    static constexpr int kMetaBytes = 32 * 4 * 2;
    static constexpr int kStepMetaBytes = 32 * 4 * 3 + 2 * 4;
    static constexpr int kStepWarp = kTwBytes + kStepMetaBytes;
    // element phase, per-warp shares of the block's regions: sample data, pair list (4 B items), c-bar
    // per thread and frequency, the rows of each evaluated pair (or a group's pass masks), meta (active
    // bits, scan sums), candidate masks; then the warps' gradient accumulators [splat][21]
    static constexpr int kSampleBytes = 32 * kSF * 4;
    static constexpr int kItemBytes = 32 * 32 * 2;
    static_assert(kGroupWords * 32 * 4 <= 32 * GR_COUNT * 4, "a group's pass masks fit in the pair-rows buffer");
    static constexpr int kCbBytes = 32 * CH * 11 * 4;
    static constexpr int kGitemBytes = 32 * GR_COUNT * 4;
    static constexpr int kCandBytes = kMaxSplatWords * 4;
    static constexpr int kFixed = kSampleBytes + kItemBytes + kCbBytes + kGitemBytes + kMetaBytes + kCandBytes;
    __host__ __device__ static size_t acc_bytes(int ntot) { return (size_t(ntot) * GR_COUNT * 4 + 15) / 16 * 16; }
    __host__ __device__ static size_t tab_bytes(int ntot) { return (size_t(ntot) * ST_COUNT * 4 + 15) / 16 * 16; }
    // the gradient accumulator is per warp in shared memory, or (large tables) the unit's own block of gunit
    __host__ __device__ static size_t warp_bytes(int ntot, bool global_acc = false) { return size_t(kFixed) + (global_acc ? 0 : acc_bytes(ntot)); }
    __host__ __device__ static size_t bytes(int ntot, int warps, bool global_acc = false) {
        return tab_bytes(ntot) + size_t(warps) * warp_bytes(ntot, global_acc);
    }
    __host__ __device__ static size_t step_bytes(int warps) { return size_t(warps) * kStepWarp; }
};

// The work unit of a persistent warp, decoded as k_consume decodes it (last rays first).
struct AdjUnit {
    long long ur, jbase, j;
    int seg, f, v0, k0, k1, nc;
    bool live, dead;
};
// The unit of warp `warp` in block work unit ub: the block's W warps take W consecutive chunks of
// 32 rays with the same segment, frame and frequencies (k_consume's block units, last rays first) and
// step through the samples together. U.ur is the warp unit's index in the numbering of the per-unit
// partial sums; a warp whose chunk lies past the last ray is dead (no rays, no partial sums).
template <int CH>
__device__ __forceinline__ AdjUnit adj_block_unit(const MixedJob& job, long long btotal, unsigned long long ub, int warp, int W, int lane,
                                                  int N) {
    AdjUnit U;
    const long long per_chunk = (long long)job.nseg * job.nframes * job.nvc;
    const long long br = btotal - 1 - (long long)ub;
    const long long wg = (br / per_chunk) * W + warp;
    const long long rem = br % per_chunk;
    U.dead = wg >= job.nchunks;
    U.ur = wg * per_chunk + rem;
    U.seg = int(rem / (job.nframes * job.nvc));
    const int y = int(rem % (job.nframes * job.nvc));
    U.f = y / job.nvc;
    U.v0 = (y % job.nvc) * CH;
    U.jbase = wg * 32;
    const long long j0 = U.jbase + lane;
    U.live = j0 < job.npix;
    U.j = U.live ? j0 : job.npix - 1;
    U.k0 = 1 + U.seg * job.seg_len;
    U.k1 = min(N + 1, U.k0 + job.seg_len);
    U.nc = min(CH, job.nfreq - U.v0);
    return U;
}

// The step phase: every block work unit walks its segment from the last sample to the first (all
// threads together), carrying T per (thread, frequency); the (thread, frequency) pairs with an active
// sample are spread over the block, each computes w_k = P_k^T w_s and the step adjoint, writes c-bar
// over the stored coefficients (fields 16..26 of its gstate row) and advances T <- E + O T.
template <int CH, int NT>
__global__ void __launch_bounds__(NT)
k_adj_steps(Spacetime st, MixedJob job, const double* __restrict__ cnu, const double* __restrict__ plan_f, const float* __restrict__ stream,
            float* __restrict__ gstate, const unsigned char* __restrict__ gact, const float* __restrict__ bnd,
            unsigned long long* __restrict__ work) {
    extern __shared__ __align__(16) unsigned char smem[];
    using AS = AdjSmem<CH>;
    constexpr int W = NT / 32;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    float* tw = reinterpret_cast<float*>(smem);                              // [c][8][NT]: w 0..3, T 4..7
    int* meta_off = reinterpret_cast<int*>(smem + W * AS::kTwBytes);         // [NT]
    unsigned* meta_bits = reinterpret_cast<unsigned*>(meta_off + NT);        // [NT]
    float* sgd_s = reinterpret_cast<float*>(meta_bits + NT);                 // [NT]: Sigma dtau of each thread's sample
    int* wsum = reinterpret_cast<int*>(sgd_s + NT);                          // [2][W]
    int scan_par = 0;
    const int N = st.N;
    const long long npad = job.npad, npix = job.npix;
    const float a = float(st.a);
    // block work units (the phase alignment of k_consume)
    __shared__ unsigned long long s_unit;
    const long long btotal = (job.nchunks + W - 1) / W * job.nseg * job.nframes * job.nvc;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_unit = atomicAdd(work, 1ull);
        __syncthreads();
        const unsigned long long u = s_unit;
        if (u >= (unsigned long long)btotal) break;
        const AdjUnit U = adj_block_unit<CH>(job, btotal, u, warp, W, lane, N);
        const long long jb = U.jbase - warp * 32;   // the block's first ray: thread o owns ray jb + o
        float Lnu[CH];
#pragma unroll
        for (int c = 0; c < CH; ++c) Lnu[c] = float(job.L / (cnu[min(U.v0 + c, job.nfreq - 1)] / kNU0));
        const float dtau_o = float(plan_f[(long long)PF_DTAU * npad + U.j]);
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            const long long combo = (long long)min(U.v0 + c, job.nfreq - 1) * job.nframes + U.f;
            const float* b = bnd + (combo * job.nseg + U.seg) * 8 * npix + U.j;
#pragma unroll
            for (int q = 0; q < 8; ++q) tw[(c * 8 + q) * NT + tid] = (U.live && c < U.nc) ? b[(long long)q * npix] : 0.f;
        }
        for (int k = U.k1 - 1; k >= U.k0; --k) {
            const float* sp = stream + (long long)(k - 1) * SM_COUNT * npad + U.j;
            unsigned actbits = 0u;
            if (U.live && (__float_as_uint(sp[SM_FLAGS * npad]) & 8u)) {
#pragma unroll
                for (int c = 0; c < CH; ++c) {
                    if (c >= U.nc) break;
                    const long long combo = (long long)(U.v0 + c) * job.nframes + U.f;
                    if (gact[(combo * N + (k - 1)) * npad + U.j]) actbits |= 1u << c;
                }
            }
            const int n2 = __popc(actbits);
            int total2;
            const int off2 = block_exscan<NT>(n2, total2, wsum, scan_par);   // a barrier: the last sample's steps are done
            if (total2 == 0) continue;
            if (actbits) {
                // Sigma dtau of this thread's sample, for the worker that takes its steps
                const float rr = sp[SM_R * npad], cth = sp[SM_CTH * npad];
                sgd_s[tid] = (rr * rr + a * a * cth * cth) * dtau_o;
            }
            meta_off[tid] = off2;
            meta_bits[tid] = actbits;
            __syncthreads();
            for (int base = 0; base < total2; base += NT) {
                const int g = base + tid;
                if (g < total2) {
                    // owner: the last thread whose first item is <= g (offsets are non-decreasing)
                    int o = 0;
#pragma unroll
                    for (int d = 256; d >= 1; d >>= 1)
                        if (o + d < NT && meta_off[o + d] <= g) o += d;
                    unsigned bits = meta_bits[o];
                    const int jj = g - meta_off[o];
                    for (int q = 0; q < jj; ++q) bits &= bits - 1;
                    const int c = __ffs(bits) - 1;
                    const long long combo = (long long)(U.v0 + c) * job.nframes + U.f;
                    float* gs = gstate + ((combo * N + (k - 1)) * 27) * npad + jb + o;
                    float Pm[16], in[11];
#pragma unroll
                    for (int q = 0; q < 16; ++q) Pm[q] = gs[q * npad];
#pragma unroll
                    for (int q = 0; q < 11; ++q) in[q] = gs[(16 + q) * npad];
                    float* twc = tw + c * 8 * NT + o;
                    float wk[4], R[4];
#pragma unroll
                    for (int s4 = 0; s4 < 4; ++s4)
                        wk[s4] = Pm[s4] * twc[0] + Pm[4 + s4] * twc[NT] + Pm[8 + s4] * twc[2 * NT] + Pm[12 + s4] * twc[3 * NT];
#pragma unroll
                    for (int s4 = 0; s4 < 4; ++s4) R[s4] = twc[(4 + s4) * NT];
                    float Lc = Lnu[0];
#pragma unroll
                    for (int cc = 1; cc < CH; ++cc) Lc = (cc == c) ? Lnu[cc] : Lc;
                    float O[16], E[4], cb[11];
                    sample_adjoint_structured(c_moments, in, Lc * sgd_s[o], wk, R, O, E, cb);
#pragma unroll
                    for (int q = 0; q < 11; ++q) gs[(16 + q) * npad] = cb[q];
                    // (owner, frequency) pairs are distinct within a sample: no other worker touches this column
#pragma unroll
                    for (int r = 0; r < 4; ++r)
                        twc[(4 + r) * NT] = E[r] + O[4 * r] * R[0] + O[4 * r + 1] * R[1] + O[4 * r + 2] * R[2] + O[4 * r + 3] * R[3];
                }
            }
        }
    }
}

// The element phase: every block work unit visits its samples (in order, all threads together); the
// threads with an active sample test the splats against the support, the passing (thread, splat)
// pairs of up to kGroupWords candidate words go into one block list and are evaluated NT at a time
// with the sample's c-bar (read back from gstate); every warp then sums the 21 rows of the 32 pairs
// its own lanes evaluated, per splat in list order, into its accumulator (a fixed partition of the
// list: deterministic sums, no block barrier inside a round); each warp unit writes its partial sums
// to gunit, and the units are added in a fixed order.
template <int CH, int NT>
__global__ void __launch_bounds__(NT, 1)
k_adj_elements(Spacetime st, MixedJob job, const float* __restrict__ tab32, const double* __restrict__ gtab, int ntot,
               const double* __restrict__ ct, const double* __restrict__ cnu, const double* __restrict__ plan_f, const float* __restrict__ stream,
               const float* __restrict__ gstate, const unsigned char* __restrict__ gact, unsigned long long* __restrict__ work,
               float* __restrict__ gunit, int global_acc, unsigned* __restrict__ err) {
    extern __shared__ __align__(16) unsigned char smem[];
    using AS = AdjSmem<CH>;
    constexpr int W = NT / 32;
    float* tab = reinterpret_cast<float*>(smem);
    // the FP32 splat table into shared memory by one bulk copy (k_consume's staging)
    __shared__ __align__(8) unsigned long long tab_bar;
    const unsigned tab_bytes = unsigned(AS::tab_bytes(ntot));
    if (tab_bytes > 0 && !stage_bulk(tab, tab32, tab_bytes, &tab_bar, job.stage_test == 0, job.stage_test ? 4096 : kStageWaitLimit)) {
        if (threadIdx.x == 0) atomicOr(err, 1u);
        return;
    }
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // the block's regions (each the sum of the warps' shares), then the warps' accumulators
    unsigned char* bb = smem + AS::tab_bytes(ntot);
    float* sf = reinterpret_cast<float*>(bb);                                            // [kSF][NT]
    unsigned* items = reinterpret_cast<unsigned*>(bb + W * AS::kSampleBytes);           // owner << 9 | splat
    float* cbs = reinterpret_cast<float*>(bb + W * (AS::kSampleBytes + AS::kItemBytes)); // [CH][11][NT]
    float* gitem = cbs + NT * CH * 11;                                                  // [item][21] | pass masks
    unsigned* meta_bits = reinterpret_cast<unsigned*>(gitem + NT * GR_COUNT);           // [NT]
    int* wsum = reinterpret_cast<int*>(meta_bits + NT);                                 // [2][W]
    unsigned* cand = reinterpret_cast<unsigned*>(reinterpret_cast<unsigned char*>(meta_bits) + W * AS::kMetaBytes) +
                     warp * kMaxSplatWords;                                             // this warp's candidates
    float* gacc_smem = reinterpret_cast<float*>(bb + W * AS::kFixed + size_t(warp) * AS::acc_bytes(ntot));   // [splat][21]
    const int item_cap = W * AS::kItemBytes / 4;
    __syncthreads();
    __shared__ float s_reach;
    const float reach2 = table_reach2(tab, ntot, &s_reach);   // samples farther out weigh no splat
    const int N = st.N;
    const long long npad = job.npad;
    const float a = float(st.a), a_sin_tho = float(st.a * sin(st.thetao));
    const long long gsz = (long long)ntot * GR_COUNT;
    const int nw = (ntot + 31) >> 5;
    int scan_par = 0;
    // block work units (the phase alignment of k_consume)
    __shared__ unsigned long long s_unit;
    const long long btotal = (job.nchunks + W - 1) / W * job.nseg * job.nframes * job.nvc;
    __shared__ float nu[CH];   // the block unit's frequencies
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_unit = atomicAdd(work, 1ull);
        __syncthreads();
        const unsigned long long u = s_unit;
        if (u >= (unsigned long long)btotal) break;
        const AdjUnit U = adj_block_unit<CH>(job, btotal, u, warp, W, lane, N);
        // the live warps (dead ones, past the last ray, are the trailing warps) evaluate and accumulate
        const int ntl = 32 * __syncthreads_count(lane == 0 && !U.dead);
        const float t_obs = float(ct[U.f]);
        if (tid < CH) nu[tid] = float(cnu[min(U.v0 + tid, job.nfreq - 1)]);   // read after the next barrier
        const float dtau = float(plan_f[(long long)PF_DTAU * npad + U.j]);
        const float alpha = float(plan_f[(long long)PF_ALPHA * npad + U.j]), beta = float(plan_f[(long long)PF_BETA * npad + U.j]);
        const float eta = float(plan_f[(long long)PF_ETA * npad + U.j]), lam = float(plan_f[(long long)PF_LAM * npad + U.j]);
        // a dead warp has no active sample: it neither zeroes nor adds to an accumulator
        float* gacc = global_acc ? gunit + (U.dead ? 0 : U.ur) * gsz : gacc_smem;
        if (!U.dead)
            for (long long q = lane; q < gsz; q += 32) gacc[q] = 0.f;
        const int nsamp = int(plan_f[(long long)PF_NSAMP * npad + U.j]);
        const int cl = job.cand_len > 0 ? job.cand_len : job.seg_len;   // the forward pass's candidate runs
        for (int k = U.k0; k < U.k1; ++k) {
            if ((k - U.k0) % cl == 0) {
                // the candidate splats of samples [k, k + cl) (as the forward pass)
                UnitBox b = unit_box_empty();
                const int ke = min(U.k1, k + cl);
                for (int kk = k; kk < ke; ++kk) {
                    const float* bp = stream + (long long)(kk - 1) * SM_COUNT * npad + U.j;
                    if (!U.live || kk > nsamp || !(__float_as_uint(bp[SM_FLAGS * npad]) & 8u)) continue;
                    const float x = bp[SM_X * npad], y = bp[SM_Y * npad], z = bp[SM_Z * npad];
                    if (x * x + y * y + z * z > reach2) continue;
                    unit_box_add(b, x, y, z, t_obs - bp[SM_T * npad]);
                }
                unit_box_reduce(b);
                unit_candidates(tab, ntot, b, lane, cand);
            }
            const float* sp = stream + (long long)(k - 1) * SM_COUNT * npad + U.j;
            const unsigned flags = __float_as_uint(sp[SM_FLAGS * npad]);
            unsigned actbits = 0u;
            if (U.live && (flags & 8u)) {
#pragma unroll
                for (int c = 0; c < CH; ++c) {
                    if (c >= U.nc) break;
                    const long long combo = (long long)(U.v0 + c) * job.nframes + U.f;
                    if (gact[(combo * N + (k - 1)) * npad + U.j]) actbits |= 1u << c;
                }
            }
            // the sample is skipped by the whole block when no thread has an active step (a barrier)
            if (!__syncthreads_or(actbits != 0u)) continue;
            float x = 0.f, yy = 0.f, z = 0.f, ts = 0.f, rho = 0.f;
            if (actbits) {
                x = sp[SM_X * npad]; yy = sp[SM_Y * npad]; z = sp[SM_Z * npad]; ts = sp[SM_T * npad];
                const float r = sp[SM_R * npad], sth = sp[SM_STH * npad], cth = sp[SM_CTH * npad];
                rho = sqrtf(x * x + yy * yy);
                SampleFrame<float> F = sample_frame(a, r, 0.f, sth, cth, eta, lam, (flags & 2u) != 0u, (flags & 4u) != 0u);
                float* mys = sf + tid;
                mys[SF_X * NT] = x; mys[SF_Y * NT] = yy; mys[SF_Z * NT] = z; mys[SF_T * NT] = ts;
                mys[SF_PU0 * NT] = F.pu[0]; mys[SF_PU1 * NT] = F.pu[1]; mys[SF_PU2 * NT] = F.pu[2]; mys[SF_PU3 * NT] = F.pu[3];
                mys[SF_PZ0 * NT] = F.pz[0]; mys[SF_PZ1 * NT] = F.pz[1]; mys[SF_PZ2 * NT] = F.pz[2]; mys[SF_PZ3 * NT] = F.pz[3];
                mys[SF_LI * NT] = F.lapse_inv; mys[SF_OL * NT] = F.om_lapse; mys[SF_SDS * NT] = F.sDS; mys[SF_MIS * NT] = F.misS;
                mys[SF_IVP * NT] = F.ivarpi;
                mys[SF_R * NT] = r; mys[SF_STH * NT] = sth; mys[SF_CTH * NT] = cth;
                mys[SF_SG * NT] = (r * r + a * a * cth * cth) * dtau;
                mys[SF_ALPHA * NT] = alpha; mys[SF_BETA * NT] = beta;
#pragma unroll
                for (int c = 0; c < CH; ++c) {
                    if (!((actbits >> c) & 1u)) continue;
                    const long long combo = (long long)(U.v0 + c) * job.nframes + U.f;
                    const float* gs = gstate + ((combo * N + (k - 1)) * 27 + 16) * npad + U.j;
#pragma unroll
                    for (int q = 0; q < 11; ++q) cbs[(c * 11 + q) * NT + tid] = gs[q * npad];
                }
            }
            meta_bits[tid] = actbits;
            const float t = t_obs - ts;
            unsigned* gmask = reinterpret_cast<unsigned*>(gitem) + tid;   // [kGroupWords][NT]
            int single_end = -1;
            for (int g0 = 0; g0 < nw;) {
                const bool single = g0 < single_end;
                const int g1 = single ? g0 + 1 : min(nw, g0 + kGroupWords);
                int n = 0;
                unsigned m1 = 0u;
                for (int wd = g0; wd < g1; ++wd) {
                    const unsigned cm = cand[wd];
                    unsigned mask = 0u;
                    if (actbits && cm) {
                        unsigned cb2 = cm;
                        while (cb2) {
                            const int b = __ffs(cb2) - 1;
                            cb2 &= cb2 - 1;
                            const float* p = tab + (wd * 32 + b) * ST_COUNT;
                            const float dr = rho - p[ST_RHO], dz = z - p[ST_CZ];
                            if (dr * dr + dz * dz > p[ST_SUPP]) continue;
                            float q;
                            if (!splat_exponent(p, t, x, yy, z, true, q)) continue;
                            if (q < kQCUT) mask |= 1u << b;
                        }
                    }
                    if (single) m1 = mask;
                    else gmask[(wd - g0) * NT] = mask;
                    n += __popc(mask);
                }
                int total;
                const int off = block_exscan<NT>(n, total, wsum, scan_par);
                if (!single && total > item_cap) { single_end = g1; continue; }
                for (int wb = 0; wb < total; wb += item_cap) {
                    if (n > 0 && off + n > wb && off < wb + item_cap) {
                        int kk = off;
                        for (int wd = g0; wd < g1; ++wd) {
                            unsigned m = single ? m1 : gmask[(wd - g0) * NT];
                            while (m) {
                                const int b = __ffs(m) - 1;
                                m &= m - 1;
                                if (kk >= wb && kk < wb + item_cap) items[kk - wb] = (unsigned(tid) << 9) | unsigned(wd * 32 + b);
                                ++kk;
                            }
                        }
                    }
                    __syncthreads();
                    // Rounds of ntl pairs over the live warps' threads; each warp then adds the 32 pairs its
                    // own lanes evaluated to its accumulator, in list order (a fixed partition of the list,
                    // so the sums are deterministic), with no block barrier inside the window.
                    const int wt = min(item_cap, total - wb);
                    for (int base = 0; base < wt; base += ntl) {
                        const int kk0 = base + tid;
                        if (tid < ntl && kk0 < wt) {
                            const unsigned it = items[kk0];
                            const int o = int(it >> 9), i = int(it & 511u);
                            element_adjoint_ool<CH, NT>(tab + i * ST_COUNT, gtab + (long long)i * GT_COUNT, sf + o, t_obs, a, a_sin_tho, nu, U.nc,
                                                        meta_bits[o], cbs + o, gitem + tid * GR_COUNT);
                        }
                        __syncwarp();
                        // four pairs at a time: their rows are read before any sum is written back; four
                        // pairs of which two share a splat go one by one (each splat's sum in list order)
                        const int lo = base + warp * 32, hi = min(wt, lo + 32);
                        if (tid < ntl && lane < GR_COUNT) {
                            int q = lo;
                            for (; q + 4 <= hi; q += 4) {
                                const int i0 = int(items[q] & 511u), i1 = int(items[q + 1] & 511u);
                                const int i2 = int(items[q + 2] & 511u), i3 = int(items[q + 3] & 511u);
                                const float* gi = gitem + (q - base) * GR_COUNT + lane;
                                const float v0 = gi[0], v1 = gi[GR_COUNT], v2 = gi[2 * GR_COUNT], v3 = gi[3 * GR_COUNT];
                                float* a0 = gacc + i0 * GR_COUNT + lane;
                                float* a1 = gacc + i1 * GR_COUNT + lane;
                                float* a2 = gacc + i2 * GR_COUNT + lane;
                                float* a3 = gacc + i3 * GR_COUNT + lane;
                                if (i0 != i1 && i0 != i2 && i0 != i3 && i1 != i2 && i1 != i3 && i2 != i3) {
                                    const float s0 = *a0 + v0, s1 = *a1 + v1, s2 = *a2 + v2, s3 = *a3 + v3;
                                    *a0 = s0; *a1 = s1; *a2 = s2; *a3 = s3;
                                } else {
                                    *a0 += v0; *a1 += v1; *a2 += v2; *a3 += v3;
                                }
                            }
                            for (; q < hi; ++q)
                                gacc[int(items[q] & 511u) * GR_COUNT + lane] += gitem[(q - base) * GR_COUNT + lane];
                        }
                        __syncwarp();
                    }
                    // the next window's items and the next group's pass masks (in gitem) are written after this
                    __syncthreads();
                }
                g0 = g1;
            }
        }
        if (!global_acc && !U.dead) {
            float* gu = gunit + U.ur * gsz;
            for (long long q = lane; q < gsz; q += 32) gu[q] = gacc[q];
        }
        __syncwarp();
    }
}

// The sum over work units in a fixed order: stage 1 adds the units of each chunk (one thread per
// gradient entry and chunk), stage 2 the chunks.
__global__ void k_unit_reduce1(const float* __restrict__ gunit, long long nunits, long long gsz, int per_chunk, double* __restrict__ part) {
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e >= gsz) return;
    const long long u0 = (long long)blockIdx.y * per_chunk, u1 = min(nunits, u0 + per_chunk);
    double s = 0.0;
    for (long long uu = u0; uu < u1; ++uu) s += gunit[uu * gsz + e];
    part[(long long)blockIdx.y * gsz + e] = s;
}
__global__ void k_unit_reduce2(const double* __restrict__ part, int nchunks, long long gsz, double* __restrict__ out) {
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e >= gsz) return;
    double s = 0.0;
    for (int ch = 0; ch < nchunks; ++ch) s += part[(long long)ch * gsz + e];
    out[e] = s;
}

}  // namespace

// ---- forward mode: J v of the image (jvp!, src/Fit/gauss_newton.jl:91-118) ---------------------------
//
// The reference runs its tails pass on parameters that carry duals along v. Here the splat table of the
// THERMAL21 splats is built as duals (each entry with its K directional derivatives), the march stays
// plain (the geodesics do not depend on the splats), and the consumer composes (P, S) on duals: the
// weight, the frame, the thermal fits, the cap, the invariants, the rotation and the exact step are
// the same templates as the forward path, instantiated on Dual<S, K>.

namespace {

using namespace ks;

// One THERMAL21 column and K tangent directions v[k * 21 + row] -> the dual table row. The cull radii
// (ST_SUPP, ST_RHO) keep their values: the cull is a threshold, not a function of the parameters.
template <class S, int K>
__global__ void k_dual_table(int nsplat, const double* __restrict__ params, const double* __restrict__ dirs, long long dir_stride,
                             const double* __restrict__ tab, const double* __restrict__ gtab, Dual<S, K>* __restrict__ dtab) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nsplat) return;
    using D = Dual<double, K>;
    const double* p = params + 21LL * i;
    D q[21];
    for (int r = 0; r < 21; ++r) {
        q[r] = D(p[r]);
        for (int k = 0; k < K; ++k) q[r].d[k] = dirs[k * dir_stride + 21LL * i + r];
    }
    const double* t0 = tab + (long long)i * ST_COUNT;
    const double* g = gtab + (long long)i * GT_COUNT;
    D o[ST_COUNT];
    for (int e = 0; e < ST_COUNT; ++e) o[e] = D(t0[e]);
    o[ST_CX] = q[0]; o[ST_CY] = q[1]; o[ST_CZ] = q[2];
    o[ST_T0] = q[10]; o[ST_OMEGA] = q[20];
    o[ST_ES1] = exp(-q[3]); o[ST_ES2] = exp(-q[4]); o[ST_ES3] = exp(-q[5]);
    const D n = sqrt(q[6] * q[6] + q[7] * q[7] + q[8] * q[8] + q[9] * q[9]);
    const D w = q[6] / n, x = q[7] / n, y = q[8] / n, z = q[9] / n;
    o[ST_R0] = 1.0 - 2.0 * (y * y + z * z); o[ST_R1] = 2.0 * (x * y - w * z); o[ST_R2] = 2.0 * (x * z + w * y);
    o[ST_R3] = 2.0 * (x * y + w * z); o[ST_R4] = 1.0 - 2.0 * (x * x + z * z); o[ST_R5] = 2.0 * (y * z - w * x);
    o[ST_R6] = 2.0 * (x * z - w * y); o[ST_R7] = 2.0 * (y * z + w * x); o[ST_R8] = 1.0 - 2.0 * (x * x + y * y);
    o[ST_INVW] = exp(-q[11]);
    o[ST_NE] = exp(q[12]);
    o[ST_TE] = exp(q[13]);
    for (int k = 0; k < K; ++k) { o[ST_F0].d[k] = g[GT_DF0] * q[13].d[k]; o[ST_KR].d[k] = g[GT_DKR] * q[13].d[k]; }
    o[ST_BMAG] = exp(q[14]);
    if (t0[ST_BZERO] == 0.0) {
        o[ST_BHX] = sin(q[15]) * cos(q[16]); o[ST_BHY] = sin(q[15]) * sin(q[16]); o[ST_BHZ] = cos(q[15]);
    }
    o[ST_U1] = q[17]; o[ST_U2] = q[18]; o[ST_U3] = q[19];
    Dual<S, K>* out = dtab + (long long)i * ST_COUNT;
    for (int e = 0; e < ST_COUNT; ++e) {
        out[e].v = S(o[e].v);
        for (int k = 0; k < K; ++k) out[e].d[k] = S(o[e].d[k]);
    }
}

// The consumer of the JVP: RadiativeTransport on the dual table (transport.jl:171-198, step.jl:347).
template <class S, int K>
struct JvpSink {
    using D = Dual<S, K>;
    const D* tab; int ntot;
    S t_obs, nu, Lnu, a, rh_lo, dtau, alpha, beta, eta, lam, a_sin_tho, slab;
    int nmax;
    int lnL_dir;      // >= 0: the direction that carries d/d(ln L) (the step length scales with L)
    S reach2 = S(3e38f);   // table_reach2: farther samples weigh no splat
    D P[16], Sv[4];
    S zprev; int wn; bool inside, crossed, zset;

    __device__ void init() {
        for (int q = 0; q < 16; ++q) P[q] = D(S((q % 5 == 0) ? 1 : 0));
        for (int q = 0; q < 4; ++q) Sv[q] = D(S(0));
        wn = 0; inside = false; crossed = false; zset = false; zprev = S(0);
    }
    __device__ void wind(S z) {   // step.jl:379-398
        if (!zset) { zprev = z; zset = true; inside = fabs(z) < slab; crossed = false; return; }
        bool inside_now = fabs(z) < slab;
        bool crossing = zprev * z < S(0);
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
    __device__ void operator()(int, const Sample<double>& s64) {
        const S r = S(s64.r), th = S(s64.theta), ph = S(s64.phi), ts = S(s64.t);
        if (!(s64.ok && r > rh_lo)) return;
        if (nmax >= 0) {
            wind(r * cos(th));
            if (wn > nmax) return;
        }
        S x, y, z, sth, cth;
        ks_coords(a, r, th, ph, x, y, z, sth, cth);
        emit(x, y, z, ts, r, sth, cth, s64.nur, s64.nutheta);
    }
    // one sample of the FP32 stream (k_stream: position, lookback time, r, sin/cos theta, flags)
    __device__ void stream_sample(bool usable, S x, S y, S z, S ts, S r, S sth, S cth, bool nur, bool nuth) {
        if (!usable) return;
        if (nmax >= 0) {
            wind(r * cth);
            if (wn > nmax) return;
        }
        emit(x, y, z, ts, r, sth, cth, nur, nuth);
    }
    __device__ void emit(S x, S y, S z, S ts, S r, S sth, S cth, bool nur, bool nuth) {
        if (x * x + y * y + z * z > reach2) return;   // no splat reaches the sample: no element, no step
        const S t = t_obs - ts;
        D in[11];
        for (int q = 0; q < 11; ++q) in[q] = D(S(0));
        bool active = false, have_frame = false;
        SampleFrame<D> F;
        const S rho = sqrt(x * x + y * y);
        for (int i = 0; i < ntot; ++i) {
            const D* p = tab + (long long)i * ST_COUNT;
            // the circle of the pattern rotation, on values first (exact: outside it the support test fails too)
            const S dr = rho - p[ST_RHO].v, dz = z - p[ST_CZ].v;
            if (dr * dr + dz * dz > p[ST_SUPP].v) continue;
            D q;
            if (!splat_exponent(p, D(t), D(x), D(y), D(z), true, q)) continue;
            const D G = exp(-q);
            if (!(G > S(kWEIGHT_CUTOFF))) continue;
            if (!have_frame) {
                const SampleFrame<S> F0 = sample_frame(a, r, S(0), sth, cth, eta, lam, nur, nuth);
                for (int k = 0; k < 4; ++k) { F.pu[k] = D(F0.pu[k]); F.pz[k] = D(F0.pz[k]); }
                F.lapse_inv = D(F0.lapse_inv); F.om_lapse = D(F0.om_lapse); F.sDS = D(F0.sDS); F.misS = D(F0.misS); F.ivarpi = D(F0.ivarpi);
                F.r = D(F0.r); F.sth = D(F0.sth); F.cth = D(F0.cth); F.a = D(F0.a);
                have_frame = true;
            }
            const LFrame<D> lf = local_frame(F, p[ST_U1], p[ST_U2], p[ST_U3], p[ST_BHX], p[ST_BHY], p[ST_BHZ], p[ST_BZERO] != S(0),
                                             D(alpha), D(beta), D(a_sin_tho));
            const D nuf = D(nu) / lf.g;
            D sbv, cbv;
            if constexpr (is_f32<S>) pitch_sc(lf.cosB, sbv, cbv);
            else { const D thb = safe_acos(lf.cosB); sbv = sin(thb); cbv = cos(thb); }
            const Coef<D> cf = thermal_cs(p[ST_NE] * G, p[ST_TE], p[ST_F0], p[ST_KR], p[ST_BMAG], nuf, sbv, cbv);
            if (!(cf.jI > S(0) || cf.aI > S(0) || cf.rQ != S(0) || cf.rV != S(0))) continue;
            const D fe = cap_factor(cf.jI, cf.jQ, cf.jV, D(S(0.99)));
            const D fa = cap_factor(cf.aI, cf.aQ, cf.aV, D(S(0.99)));
            const D nh = nuf / S(kNU0);
            const D i2 = D(S(1)) / (nh * nh);
            const D s2c = lf.s2c, c2c = lf.c2c;
            const D jQ = cf.jQ * fe * i2, aQ = cf.aQ * fa * nh, rQ = cf.rQ * nh;
            in[0] += cf.jI * i2; in[1] += jQ * c2c; in[2] += jQ * s2c; in[3] += cf.jV * fe * i2;
            in[4] += nh * cf.aI; in[5] += aQ * c2c; in[6] += aQ * s2c; in[7] += cf.aV * fa * nh;
            in[8] += rQ * c2c; in[9] += rQ * s2c; in[10] += nh * cf.rV;
            active = true;
        }
        if (!active) return;
        const S Sg = r * r + a * a * cth * cth;
        D Dl(Lnu * Sg * dtau);
        if (lnL_dir >= 0) Dl.d[lnL_dir] = Dl.v;
        D O[16], E[4];
        transfer_step(c_moments, in, in + 4, in + 8, Dl, O, E);
        D Pn[16];
        for (int rr = 0; rr < 4; ++rr) {
            Sv[rr] += P[4 * rr] * E[0] + P[4 * rr + 1] * E[1] + P[4 * rr + 2] * E[2] + P[4 * rr + 3] * E[3];
            for (int q = 0; q < 4; ++q)
                Pn[4 * rr + q] = P[4 * rr] * O[q] + P[4 * rr + 1] * O[4 + q] + P[4 * rr + 2] * O[8 + q] + P[4 * rr + 3] * O[12 + q];
        }
        for (int q = 0; q < 16; ++q) P[q] = Pn[q];
    }
};

// One thread per (ray, combination): the image's K directional derivatives (sorted order)
// out[((d * ncombo + c) * npix + j) * 4 + s], and the image itself in img.
template <class S, int K>
__global__ void __launch_bounds__(64) k_jvp(PlanView P, Spacetime st, long long npix, const Dual<S, K>* __restrict__ dtab, int ntot,
                                            const double* __restrict__ ct, const double* __restrict__ cnu, int ncombo, double L, int nmax,
                                            double slab, double* __restrict__ img, double* __restrict__ out, int lnL_dir) {
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= npix * ncombo) return;
    const long long j = idx % npix;
    const int c = int(idx / npix);
    MarchRay<double> R = load_ray<double>(P, st, j);
    JvpSink<S, K> sink;
    sink.tab = dtab; sink.ntot = ntot;
    sink.t_obs = S(ct[c]); sink.nu = S(cnu[c]);
    const double nh = cnu[c] / kNU0;
    sink.Lnu = S(L / nh);
    sink.a = S(st.a); sink.rh_lo = S(st.rh * (1 + 1e-3)); sink.dtau = S(R.dtau);
    sink.alpha = S(P.get(PF_ALPHA, j)); sink.beta = S(P.get(PF_BETA, j)); sink.eta = S(R.eta); sink.lam = S(R.lam);
    sink.a_sin_tho = S(st.a * sin(st.thetao)); sink.slab = S(slab); sink.nmax = nmax;
    sink.lnL_dir = lnL_dir;
    sink.init();
    double rt, rp;
    march(P, st, j, R, sink, rt, rp);
    const double n3 = nh * nh * nh;
    for (int s = 0; s < 4; ++s) {
        img[(c * npix + j) * 4 + s] = double(sink.Sv[s].v) * n3;
        for (int d = 0; d < K; ++d) out[(((long long)d * ncombo + c) * npix + j) * 4 + s] = double(sink.Sv[s].d[d]) * n3;
    }
}

// The mixed J v over the FP32 sample stream of k_stream (the FP64 march rounded to FP32, the
// Kerr-Schild position formed there: the samples k_jvp<float, K> would round its own march to) instead
// of a march per thread; one thread per (ray, combination), outputs as k_jvp. At most 128 registers
// (16 warps per SM instead of 12 at 168; 4% faster on configuration-5 sets, the same J v).
template <int K>
__global__ void __launch_bounds__(64, 8) k_jvp_stream(PlanView P, Spacetime st, long long npix, const Dual<float, K>* __restrict__ dtab, int ntot,
                                                   const double* __restrict__ ct, const double* __restrict__ cnu, int ncombo, double L, int nmax,
                                                   double slab, const float* __restrict__ stream, double* __restrict__ img, double* __restrict__ out,
                                                   int lnL_dir) {
    __shared__ float s_reach;
    const float reach2 = table_reach2(dtab, ntot, &s_reach);   // before any thread leaves: it has block barriers
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= npix * ncombo) return;
    const long long j = idx % npix;
    const int c = int(idx / npix);
    const long long npad = P.npad;
    JvpSink<float, K> sink;
    sink.tab = dtab; sink.ntot = ntot; sink.reach2 = reach2;
    sink.t_obs = float(ct[c]); sink.nu = float(cnu[c]);
    const double nh = cnu[c] / kNU0;
    sink.Lnu = float(L / nh);
    sink.a = float(st.a); sink.rh_lo = float(st.rh * (1 + 1e-3)); sink.dtau = float(P.get(PF_DTAU, j));
    sink.alpha = float(P.get(PF_ALPHA, j)); sink.beta = float(P.get(PF_BETA, j));
    sink.eta = float(P.get(PF_ETA, j)); sink.lam = float(P.get(PF_LAM, j));
    sink.a_sin_tho = float(st.a * sin(st.thetao)); sink.slab = float(slab); sink.nmax = nmax;
    sink.lnL_dir = lnL_dir;
    sink.init();
    const int Nj = int(P.get(PF_NSAMP, j));
    const float* sp = stream + j;
    for (int k = 1; k <= Nj; ++k, sp += SM_COUNT * npad) {
        const unsigned flags = __float_as_uint(sp[SM_FLAGS * npad]);
        sink.stream_sample((flags & 8u) != 0u, sp[SM_X * npad], sp[SM_Y * npad], sp[SM_Z * npad], sp[SM_T * npad], sp[SM_R * npad],
                           sp[SM_STH * npad], sp[SM_CTH * npad], (flags & 2u) != 0u, (flags & 4u) != 0u);
    }
    const double n3 = nh * nh * nh;
    for (int s = 0; s < 4; ++s) {
        img[(c * npix + j) * 4 + s] = double(sink.Sv[s].v) * n3;
        for (int d = 0; d < K; ++d) out[(((long long)d * ncombo + c) * npix + j) * 4 + s] = double(sink.Sv[s].d[d]) * n3;
    }
}

}  // namespace

namespace {

// A = J^T J (normal_matrix, gauss_newton.jl:486-494) of a row-major m x n FP64 Jacobian, FP64 tiles
// of 32 x 32 with the shared k-slab; only the upper triangle's tiles are computed and mirrored.
__global__ void k_normal_fp64(long long m, int n, const double* __restrict__ J, double* __restrict__ A) {
    __shared__ double Ja[32][33], Jb[32][33];
    const int bi = blockIdx.y, bj = blockIdx.x;
    if (bj < bi) return;
    const int tx = threadIdx.x, ty = threadIdx.y;   // 32 x 8
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (long long k0 = 0; k0 < m; k0 += 32) {
        for (int q = 0; q < 4; ++q) {
            const int kk = ty + 8 * q;
            const long long r = k0 + kk;
            const int ca = bi * 32 + tx, cb = bj * 32 + tx;
            Ja[kk][tx] = (r < m && ca < n) ? J[r * n + ca] : 0.0;
            Jb[kk][tx] = (r < m && cb < n) ? J[r * n + cb] : 0.0;
        }
        __syncthreads();
        for (int kk = 0; kk < 32; ++kk) {
            const double b = Jb[kk][tx];
            for (int q = 0; q < 4; ++q) acc[q] += Ja[kk][ty + 8 * q] * b;
        }
        __syncthreads();
    }
    for (int q = 0; q < 4; ++q) {
        const int i = bi * 32 + ty + 8 * q, j = bj * 32 + tx;
        if (i < n && j < n) { A[(long long)i * n + j] = acc[q]; A[(long long)j * n + i] = acc[q]; }
    }
}

// row-major m x n (double) -> the split GEMM operand y[n][ld] (row c holds column c of x)
__global__ void k_transpose_split(long long m, int n, const double* __restrict__ x, float* __restrict__ hi, float* __restrict__ lo,
                                  long long ld) {
    __shared__ float t[32][33];
    const long long r0 = (long long)blockIdx.y * 32;
    const int c0 = blockIdx.x * 32;
    for (int q = threadIdx.y; q < 32; q += blockDim.y) {
        const long long r = r0 + q;
        const int cc = c0 + threadIdx.x;
        t[q][threadIdx.x] = (r < m && cc < n) ? float(x[r * n + cc]) : 0.f;
    }
    __syncthreads();
    for (int q = threadIdx.y; q < 32; q += blockDim.y) {
        const int cc = c0 + q;
        const long long r = r0 + threadIdx.x;
        if (cc < n && r < m) ksdft::split_store(hi, lo, (long long)cc * ld + r, t[threadIdx.x][q]);
    }
}
__global__ void k_to_f64(long long n, const float* __restrict__ x, double* __restrict__ y) {
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q < n) y[q] = double(x[q]);
}

}  // namespace
