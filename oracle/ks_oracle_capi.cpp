// ks_oracle_capi.cpp -- C entry points of the CPU oracle, for ctypes in tests/ and the CPU-baseline
// leg of bench.py. TEST INFRASTRUCTURE ONLY: the CUDA library never links this.
//
// Every image entry point works in screen order (pixel i of the camera), one ray per OpenMP
// iteration, dynamic schedule (rays differ in cost by root case).
#include "ks_transfer.hpp"
#include <cstring>
#ifdef _OPENMP
#include <omp.h>
#endif

using namespace kso;

extern "C" {

int kso_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void kso_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

// Per-ray constants: out is npix x 24 (row per pixel):
// eta, lam, numreals, k, c, fo, tau_total, tau_valid, Gtheta_o, r1re, r1im, r2re, r2im, r3re, r3im,
// r4re, r4im, pmu, pscale, tempfac, poffset, Manchor(M=64), K2, scattering
void kso_ray_constants(double a, double thetao, const double* alpha, const double* beta, long npix, double* out) {
#pragma omp parallel for schedule(dynamic, 64)
    for (long i = 0; i < npix; ++i) {
        Ray R = make_ray(a, thetao, alpha[i], beta[i]);
        double* o = out + 24 * i;
        o[0] = R.eta; o[1] = R.lam; o[2] = R.roots.numreals; o[3] = R.k; o[4] = R.c; o[5] = R.fo;
        o[6] = R.tau_total; o[7] = R.tau_valid; o[8] = R.Gtheta_o;
        for (int q = 0; q < 4; ++q) { o[9 + 2 * q] = R.roots.r[q].real(); o[10 + 2 * q] = R.roots.r[q].imag(); }
        o[17] = R.pmu; o[18] = R.pscale; o[19] = R.tempfac; o[20] = R.poffset;
        o[21] = anchor_interval(64, 1.0 - R.k); o[22] = R.K2; o[23] = R.scattering ? 1.0 : 0.0;
    }
}

// The sample stream of the recurrence march (quadrature.jl:231-296): arrays npix x N, row per pixel.
// flags: bit 0 ok, bit 1 nu_r, bit 2 nu_theta (direct_march.jl:14-17).
void kso_march_samples(double a, double thetao, const double* alpha, const double* beta, long npix, int N, int M,
                       double* t, double* r, double* th, double* ph, unsigned char* flags, double* resid_t, double* resid_phi) {
#pragma omp parallel for schedule(dynamic, 16)
    for (long i = 0; i < npix; ++i) {
        Ray R = make_ray(a, thetao, alpha[i], beta[i]);
        size_t base = size_t(i) * N;
        march_ray(R, N, M, [&](int k, const Sample& s) {
            size_t q = base + (k - 1);
            t[q] = s.t; r[q] = s.r; th[q] = s.theta; ph[q] = s.phi;
            flags[q] = (s.ok ? 1 : 0) | (s.nur ? 2 : 0) | (s.nutheta ? 4 : 0);
        }, resid_t + i, resid_phi + i);
    }
}

// t~ and phi from the anchor evaluator at every sample k = 1..N (no recurrence): npix x N.
void kso_anchor_values(double a, double thetao, const double* alpha, const double* beta, long npix, int N,
                       double* t, double* ph, unsigned char* ok) {
#pragma omp parallel for schedule(dynamic, 4)
    for (long i = 0; i < npix; ++i) {
        Ray R = make_ray(a, thetao, alpha[i], beta[i]);
        double dtau = mino_step(R.tau_total, N);
        std::vector<Anchor> A = ray_anchors(R, N, 1, dtau);
        for (int k = 0; k < N; ++k) {
            t[size_t(i) * N + k] = A[k].t; ph[size_t(i) * N + k] = A[k].phi; ok[size_t(i) * N + k] = A[k].ok;
        }
    }
}

// Thin image (Splats.jl:113-147), params 14 x nsplat column-major, out[npix] screen order.
void kso_thin_image(double a, double thetao, const double* alpha, const double* beta, long npix, int N, int M,
                    const double* params, int nsplat, double t_obs, double* out, double* resid_t, double* resid_phi) {
#pragma omp parallel for schedule(dynamic, 16)
    for (long i = 0; i < npix; ++i) {
        Ray R = make_ray(a, thetao, alpha[i], beta[i]);
        out[i] = thin_ray(R, N, M, params, nsplat, t_obs, resid_t ? resid_t + i : nullptr, resid_phi ? resid_phi + i : nullptr);
    }
}

// Polarized image (polarized.jl:160-179) of nsets splat sets (a composite model, transport.jl:348-358).
// kinds/nrows/nsplat/params describe each set; hyp (kappa sets) per set may be null; knots for KNOT21.
// out is npix x 4 (I, Q, U, V in cgs), screen order.
void kso_polarized_image(double a, double thetao, const double* alpha, const double* beta, long npix, int N, int M,
                         int nsets, const int* kinds, const int* nrows, const int* nsplat, const double* const* params,
                         const double* const* hyp, const double* const* knots, const double* const* knot_times, const int* nknots,
                         double gmax, double t_obs, double nu, double L, int nmax, double slab, double* out) {
    std::vector<SplatSet> sets(nsets);
    for (int s = 0; s < nsets; ++s) {
        sets[s].kind = kinds[s]; sets[s].nrows = nrows[s]; sets[s].nsplat = nsplat[s]; sets[s].params = params[s];
        sets[s].gmax = gmax;
        sets[s].hyp = hyp ? hyp[s] : nullptr;
        sets[s].knots = knots ? knots[s] : nullptr;
        sets[s].knot_times = knot_times ? knot_times[s] : nullptr;
        sets[s].nknots = nknots ? nknots[s] : 0;
    }
#pragma omp parallel for schedule(dynamic, 4)
    for (long i = 0; i < npix; ++i) {
        Ray R = make_ray(a, thetao, alpha[i], beta[i]);
        PolarizedResult res = polarized_ray(R, N, M, sets, t_obs, nu, L, nmax, slab);
        out[4 * i] = res.I; out[4 * i + 1] = res.Q; out[4 * i + 2] = res.U; out[4 * i + 3] = res.V;
    }
}

// ipole's RIAF (test/riaf_model.jl) through the RadiativeTransport consumer at one frequency
// (stokes_image, test/test_polarized.jl:54-61): out npix x 4 (I, Q, U, V in cgs), screen order.
// mirror_chi != 0 plants a sign error in the screen angle (for the tests of the comparison itself).
void kso_riaf_image(double a, double thetao, const double* alpha, const double* beta, long npix, int N, int M, int pandya,
                    double nu, double L, int mirror_chi, double* out) {
    RIAF m = riaf_example(a, pandya != 0);
#pragma omp parallel for schedule(dynamic, 4)
    for (long i = 0; i < npix; ++i) {
        Ray R = make_ray(a, thetao, alpha[i], beta[i]);
        PolarizedResult res = riaf_ray(R, N, M, m, nu, L, mirror_chi != 0);
        out[4 * i] = res.I; out[4 * i + 1] = res.Q; out[4 * i + 2] = res.U; out[4 * i + 3] = res.V;
    }
}

// The exact step (step.jl:27-54): O (4x4 row-major) and E = Ej j.
void kso_transfer_step(const double* j, const double* alpha, const double* rho, double D, double* O, double* E) {
    V4 jj = {j[0], j[1], j[2], j[3]}, al = {alpha[0], alpha[1], alpha[2], alpha[3]};
    M4 Om; V4 Ev;
    transfer_step(jj, al, rho, D, Om, Ev);
    std::memcpy(O, Om.data(), 16 * sizeof(double));
    std::memcpy(E, Ev.data(), 4 * sizeof(double));
}

// Coefficient fits on vectors (coefficients.jl, kappa.jl): out is n x 8 (jI jQ jV aI aQ aV rQ rV).
void kso_thermal(long n, const double* ne, const double* Te, const double* B, const double* nu, const double* th, int dexter_rhoV, int pandya,
                 double* out) {
    for (long i = 0; i < n; ++i) {
        Coeffs c = thermal_synchrotron(ne[i], Te[i], B[i], nu[i], th[i], dexter_rhoV != 0, pandya != 0);
        double v[8] = {c.jI, c.jQ, c.jV, c.aI, c.aQ, c.aV, c.rQ, c.rV};
        std::memcpy(out + 8 * i, v, sizeof v);
    }
}
void kso_powerlaw(long n, const double* ne, const double* p, const double* gmin, const double* gmax, const double* B, const double* nu,
                  const double* th, double* out) {
    for (long i = 0; i < n; ++i) {
        Coeffs c = powerlaw_synchrotron(ne[i], p[i], gmin[i], gmax[i], B[i], nu[i], th[i]);
        double v[8] = {c.jI, c.jQ, c.jV, c.aI, c.aQ, c.aV, c.rQ, c.rV};
        std::memcpy(out + 8 * i, v, sizeof v);
    }
}
void kso_kappa(long n, const double* ne, const double* kap, const double* w, const double* B, const double* nu, const double* th,
               const double* hyp, double* out) {
    for (long i = 0; i < n; ++i) {
        Coeffs c = kappa_synchrotron(ne[i], kap[i], w[i], B[i], nu[i], th[i], hyp[i]);
        double v[8] = {c.jI, c.jQ, c.jV, c.aI, c.aQ, c.aV, c.rQ, c.rV};
        std::memcpy(out + 8 * i, v, sizeof v);
    }
}
void kso_besselk01(long n, const double* x, double* k0, double* k1) {
    for (long i = 0; i < n; ++i) besselk01(x[i], k0[i], k1[i]);
}
void kso_jacobi_state(long n, const double* u, const double* m, double* sn, double* cn, double* dn) {
    for (long i = 0; i < n; ++i) { JState s = jacobi_state(u[i], m[i]); sn[i] = s.sn; cn[i] = s.cn; dn[i] = s.dn; }
}
void kso_ellipf(long n, const double* phi, const double* m, double* out) {
    for (long i = 0; i < n; ++i) out[i] = ellipf(phi[i], m[i]);
}
// Local frame (frames.jl:108-128): out = (g, cos theta_B, chi) per input row.
void kso_local_frame(long n, double a, double thetao, const double* r, const double* th, const double* eta, const double* lam,
                     const unsigned char* nur, const unsigned char* nuth, const double* alpha, const double* beta,
                     const double* u, const double* B, double* out) {
    for (long i = 0; i < n; ++i) {
        Frame f = local_frame(a, r[i], th[i], eta[i], lam[i], nur[i] != 0, nuth[i] != 0, alpha[i], beta[i], thetao, u + 3 * i, B + 3 * i);
        out[3 * i] = f.g; out[3 * i + 1] = f.cosB; out[3 * i + 2] = f.chi;
    }
}

}  // extern "C"
