/*
 * kerrsplat_b200.h -- C ABI of libkerrsplat_b200.so, the B200 (sm_100a) render hot path of
 * KerrSplat: per-pixel geodesic constants sorted by radial root case, the fused Recurrence(M)
 * geodesic march (Jacobi addition-theorem recurrence for r and theta, anchored Mino-time
 * quadrature for t~ and phi) and the transport consumers folded over it.
 *
 * Conventions (all entry points):
 *   - every call returns an int status (KS_OK = 0); nothing throws across the ABI, and
 *     ks_last_error(ctx) holds a one-line message for the last failure;
 *   - calls are synchronous: they return after the device work is complete;
 *   - array arguments may be host or device pointers (the library asks the CUDA runtime which);
 *     host arrays are staged through the library's own device buffers;
 *   - the library owns the per-ray constants, the anchor table and its scratch buffers; the
 *     caller owns inputs and outputs;
 *   - a context is not thread-safe: one context per host thread, or external locking.
 *
 * Each declaration cites the reference (KerrSplat.jl) entry point it replaces, by file:line
 * within the reference project.
 */
#ifndef KERRSPLAT_B200_H
#define KERRSPLAT_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define KS_OK 0
#define KS_ERR_ARGUMENT 1         /* bad size or argument (reference: ArgumentError / DimensionMismatch) */
#define KS_ERR_NOT_REGENERATED 2  /* render before ks_regenerate (reference: cache.jl:203) */
#define KS_ERR_OUT_OF_MEMORY 3
#define KS_ERR_NONFINITE 4        /* NaN/Inf in an input */
#define KS_ERR_DEVICE 5           /* CUDA error */
#define KS_ERR_TIMEOUT 6          /* a bounded device wait gave up */

/* precision of a render */
#define KS_FP64 0   /* the plain FP64 path: one re-march per (frame, frequency), like the reference */
#define KS_MIXED 1  /* FP64 ray constants and anchors; the march once per render in FP32 (the radial
                       recurrence and the quadrature, re-anchored to the FP64 anchors every M samples;
                       the polar state, cos theta and krang_visible in FP64); the FP32 transport
                       (coefficients, frames, the exact step) */
#define KS_MIXED_GEO64 2  /* ks_render, the adjoint and J v: the FP64 march feeding the same FP32 transport
                             (the reference's precision(cache, Float32) arrangement, cache.jl:212-232) */

/* output order */
#define KS_ORDER_SORTED 0   /* root-case-sorted slots (the reference's fused_march! output) */
#define KS_ORDER_SCREEN 1   /* camera order (the reference's to_screen/unsort, cache.jl:271-296) */

/* splat parameter layouts (column-major nrows x nsplat) */
#define KS_THIN14 0       /* Splats.jl:54 */
#define KS_THERMAL21 1    /* polarized.jl:17-19 */
#define KS_POWERLAW22 2   /* populations.jl:13-15 */
#define KS_KAPPA22 3      /* populations.jl:24-26 */
#define KS_KNOT21 4       /* trajectories.jl:80-88: THERMAL21 rows with centres from knots */

typedef struct ks_context ks_context;

/* One splat set of a scene (a Transfer model; several sets form a CompositeModel,
 * transport.jl:348-358). */
typedef struct ks_splat_set {
    int32_t kind;              /* KS_THERMAL21, KS_POWERLAW22, KS_KAPPA22, KS_KNOT21 */
    int32_t nsplat;
    const double* params;      /* nrows(kind) x nsplat, column-major */
    const double* hyp;         /* KS_KAPPA22: per-splat 2F1 factor (kappa.jl:97-100); else NULL */
    const double* knots;       /* KS_KNOT21: 3 x nknots x nsplat knot centres; else NULL */
    const double* knot_times;  /* KS_KNOT21: nknots increasing coordinate times */
    int32_t nknots;
    double gamma_max;          /* KS_POWERLAW22: gamma_max of the set (populations.jl:40) */
} ks_splat_set;

/* Context (the device-side GeodesicCache, cache.jl:85-125, without the Julia object). */
int ks_context_create(int device, int flags, ks_context** out);
int ks_context_destroy(ks_context* ctx);
const char* ks_last_error(const ks_context* ctx);

/* Camera (camera.jl:19-46 / GeodesicCache(backend, camera, Val(N)), cache.jl:106-125):
 * npix screen points, screen shape (nalpha, nbeta) with nalpha * nbeta == npix. */
int ks_camera_set(ks_context* ctx, const double* alpha, const double* beta, int64_t npix,
                  int32_t nalpha, int32_t nbeta);

/* regenerate!(cache, a, theta_o; marcher = Fused(M)) (cache.jl:153-180): root cases, the stable
 * case sort (4, 2, 0 real roots), the FP64 per-ray constants and the FP64 anchor table of every
 * ray for `nsamples` samples and anchor interval `anchor_M` (Recurrence(M)/Fused(M)). */
int ks_regenerate(ks_context* ctx, double a, double theta_o, int32_t nsamples, int32_t anchor_M);

/* regenerate! with a sample count per ray: ray j gets N_j = clamp(64 ceil(samples_per_mino tau_total_j / 64),
 * nmin, nmax) samples at tau_k = k tau_total_j / (N_j + 1), k = 1..N_j, i.e. exactly the samples of a
 * uniform-N run with N = N_j for that ray (the reference runs mixed counts as uniform-N tiles,
 * tiles(), cache.jl:241-246). Every other entry point follows each ray's own count. */
int ks_regenerate_uneven(ks_context* ctx, double a, double theta_o, double samples_per_mino, int32_t nmin, int32_t nmax,
                         int32_t anchor_M);

/* The sample count of every ray (sorted order), npix int32. */
int ks_get_nsamples(ks_context* ctx, int32_t* nsamples);

/* cache.perm / cache.ranges (cache.jl:73-76, pixel_constants.jl:167-176): perm[j] is the screen
 * index (0-based) of sorted slot j; ranges = {case2_begin, case2_end, case3_begin, case3_end,
 * case4_begin, case4_end} as half-open 0-based slot ranges. */
int ks_get_perm(ks_context* ctx, int64_t* perm);
int ks_get_ranges(ks_context* ctx, int64_t ranges[6]);

/* cache.residual_t / residual_phi (cache.jl:78-79): the largest |quadrature - anchor| of each ray
 * in the last FP64 march (sorted order). */
int ks_get_residuals(ks_context* ctx, double* resid_t, double* resid_phi);

/* Per-ray constants in sorted order, npix x 24 rows (PixelConstants, pixel_constants.jl:29-54,
 * with the march constants): eta, lambda, numreals, k, c, fo (I0_inf), tau_total, tau_valid,
 * G_theta^o, r1..r4 (re, im), mu_theta, scale_theta, tempfac, offset_theta, M_anchor, 2K, scattering. */
int ks_get_ray_constants(ks_context* ctx, double* out);

/* Recurrence(M) stored mode (quadrature_march!, quadrature.jl:336-348): every sample of every ray,
 * npix x nsamples arrays in sorted order; flags bit 0 ok, bit 1 nu_r, bit 2 nu_theta
 * (direct_march.jl:14-17). */
int ks_march_samples(ks_context* ctx, double* t, double* r, double* theta, double* phi, uint8_t* flags);

/* thin_image!(out, cache, params, t_obs) (Splats.jl:137-140): optically-thin Stokes I of
 * KS_THIN14 splats at one observation time; out[npix] in `order`. */
int ks_thin_image(ks_context* ctx, const double* params, int32_t nsplat, double t_obs, int32_t precision,
                  double* out, int32_t order);

/* polarized_image! / polarized_cube (polarized.jl:160-198) over frames x frequencies:
 * out has npix x 4 x nframes x nfreq doubles, index ((f_nu * nframes + f_t) * npix + pixel) * 4 + stokes,
 * Stokes (I, Q, U, V) in cgs (observed_stokes, transport.jl:337), pixels in `order`.
 * nmax >= 0 truncates rays after their nmax-th passage through |z| < slab (transport.jl:182-188). */
int ks_render(ks_context* ctx, const ks_splat_set* sets, int32_t nsets, const double* times, int32_t nframes,
              const double* nus, int32_t nfreq, double L, int32_t precision, int32_t nmax, double slab,
              double* out, int32_t order);

/* ipole's RIAF through the polarized consumer: the fluid model of test/riaf_model.jl:11-93 (the reference's
 * RIAFModel, rendered by stokes_image = fused_march!(RadiativeTransport(model, nu, L), out, cache),
 * test/test_polarized.jl:54-61) at nfreq frequencies. model = {nth0, Te0, disk_h, pow_nth, pow_T, Ne_unit,
 * Te_unit, eps, r_isco, rout} (riaf_example, riaf_model.jl:31-34); pandya != 0 selects the Pandya
 * emissivities (ipole's emission_type 1). out has npix x 4 x nfreq doubles, index (f_nu * npix + pixel) * 4
 * + stokes, in cgs, pixels in `order`. KS_FP64 runs the element and the step in FP64, KS_MIXED in FP32
 * (the march stays FP64 in both). */
#define KS_RIAF_PARAMS 10
int ks_riaf_image(ks_context* ctx, const double* model, int32_t pandya, const double* nus, int32_t nfreq, double L, int32_t precision,
                  double* out, int32_t order);

/* Visibilities of an image (vis_kernel!, src/Fit/device_visibilities.jl:61-73): `image` npix x 4
 * (Stokes I, Q, U, V per pixel, in `order`), V nuv x 4 complex as (re, im) doubles,
 * V_k = tap_k scale sum_j I_j exp(2 pi i (u_k l_j + v_k m_j)) with l = -(i - (nalpha + 1)/2) psize
 * (east is -alpha), m = (j - (nbeta + 1)/2) psize; tap may be NULL (ones). KS_FP64: the direct
 * transform; KS_MIXED: the separable transform as 3xTF32 tensor-core GEMMs. */
int ks_visibilities(ks_context* ctx, const double* image, int32_t order, int64_t nuv, const double* u, const double* v,
                    const double* tap, double psize, double scale, int32_t precision, double* V);

/* The adjoint transform (seed_kernel!, device_visibilities.jl:76-88): seed_j = sum_k Re[w_k conj(dV_k/dI_j)]
 * for weights w (nuv x 4 complex); seed npix x 4 in `order`. */
int ks_vis_seed(ks_context* ctx, const double* w, int64_t nuv, const double* u, const double* v, const double* tap,
                double psize, double scale, int32_t precision, double* seed, int32_t order);

/* frame_chi2_seed! (device_visibilities.jl:97-111): chi^2 = sum |(g V - d)/sigma|^2 over baselines and
 * Stokes, and the seed of the weights 2 conj(g) r / sigma; g (nuv complex) may be NULL (no gains),
 * vis nuv x 4 complex, sigma nuv x 4. */
int ks_frame_chi2_seed(ks_context* ctx, const double* image, int32_t order, int64_t nuv, const double* u, const double* v,
                       const double* tap, const double* g, const double* vis, const double* sigma, double psize, double scale,
                       int32_t precision, double* chi2, double* seed);

/* The gradient of l = sum dstokes . Stokes with respect to every splat parameter (the dual sweep:
 * polarized_tails! + polarized_dual_sweep!, src/Splats/dual_gradient.jl:190-249, as driven by
 * sweep_passes, src/Fit/Fit.jl:451-485). Thermal polarized splats (KS_THERMAL21) only, as in the
 * reference. dstokes has the layout of ks_render's out (npix x 4 x nframes x nfreq, pixels in
 * `order`), the adjoint of the observed Stokes vectors in cgs. dparams receives 21 x nsplat per set,
 * column-major, the sets concatenated; with `accumulate` the gradient is added to it. KS_FP64 runs
 * the reference's structure (stored FP64 samples, backward tails, forward duals, per-ray slots);
 * KS_MIXED the FP32 transport with a per-segment reverse pass. Deterministic: no atomics. */
int ks_adjoint(ks_context* ctx, const ks_splat_set* sets, int32_t nsets, const double* times, int32_t nframes, const double* nus,
               int32_t nfreq, double L, int32_t precision, int32_t nmax, double slab, const double* dstokes, int32_t order,
               double* dparams, int32_t accumulate);

/* chi2_gradient! (src/Fit/Fit.jl:502-534) with the image-domain residuals of _frame_seed! (Fit.jl:537-577):
 * chi^2 = sum over unmasked pixels, Stokes and (frame, frequency) of ((image - data) / sigma)^2 and
 * its gradient, in one forward and one reverse pass. data and sigma have the layout of ks_render's out
 * in screen order (sigma may be NULL: then sigma_scalar for every entry); mask (npix x nframes x nfreq
 * bytes, screen order, nonzero = used) may be NULL. chi2 (one double), image (optional, screen order)
 * and dparams (as ks_adjoint) are outputs. */
int ks_chi2_gradient(ks_context* ctx, const ks_splat_set* sets, int32_t nsets, const double* times, int32_t nframes, const double* nus,
                     int32_t nfreq, double L, int32_t precision, int32_t nmax, double slab, const double* data, const double* sigma,
                     double sigma_scalar, const uint8_t* mask, double* chi2, double* dparams, int32_t accumulate, double* image);

/* The visibility chi^2 of one frame and its gradient (timeresolved_gradient!'s device path,
 * src/Fit/timeresolved.jl:115-138: the forward image, frame_chi2_seed!, device_visibilities.jl:97-111,
 * and the reverse pass seeded by the adjoint transform), in one forward and one reverse pass: nuv
 * baselines (u, v, tap, gains g as in ks_frame_chi2_seed; vis nuv x 4 complex, sigma nuv x 4), the DFT in
 * the render's precision class (KS_MIXED: 3xTF32 tensor cores). chi2, dparams (as ks_adjoint) and the
 * image (optional, screen order) are outputs. */
int ks_vis_chi2_gradient(ks_context* ctx, const ks_splat_set* sets, int32_t nsets, double t_obs, double nu, double L, int32_t precision,
                         int32_t nmax, double slab, int64_t nuv, const double* u, const double* v, const double* tap, const double* g,
                         const double* vis, const double* sigma, double psize, double scale, double* chi2, double* dparams,
                         int32_t accumulate, double* image);

/* J v of the image (jvp!, src/Fit/gauss_newton.jl:91-118, whose tails pass runs on parameters carrying
 * duals along v): the directional derivatives of the observed Stokes images along ndir directions
 * `dirs` (ndir x nparams, each direction laid out like dparams of ks_adjoint), into dimage
 * (ndir x nfreq x nframes x npix x 4, pixels in `order`; the image itself into `image` when not NULL).
 * Thermal polarized splats only; KS_FP64 carries FP64 duals, KS_MIXED FP32 duals; eight directions per
 * pass (jacobian!'s chunk, gauss_newton.jl:432-479). */
int ks_jvp(ks_context* ctx, const ks_splat_set* sets, int32_t nsets, const double* times, int32_t nframes, const double* nus,
           int32_t nfreq, double L, int32_t precision, int32_t nmax, double slab, const double* dirs, int32_t ndir, double* dimage,
           int32_t order, double* image);

/* The image's derivatives with respect to the spacetime block (a, theta_o, ln L) that
 * spacetime_valgrad (src/Fit/joint.jl:74-82) takes with three-partial duals through regenerate! and the
 * transport: dimage (3 x nfreq x nframes x npix x 4, screen order) = d/da, d/dtheta_o, d/d(ln L) of the
 * observed Stokes images, exact forward-mode duals through the ray constants, the Mino step, the anchors,
 * the recurrence march and the polarized consumer (all splat kinds, knot splats included) at the
 * context's sample counts, anchor spacing and sorted order. The pass runs in FP64 duals for either
 * precision. image (optional, screen order): the image of the same pass. The context is not changed. */
int ks_spacetime_derivatives(ks_context* ctx, const ks_splat_set* sets, int32_t nsets, const double* times, int32_t nframes,
                             const double* nus, int32_t nfreq, double L, int32_t precision, int32_t nmax, double slab, double* dimage,
                             double* image);

/* normal_matrix(J) (src/Fit/gauss_newton.jl:486-494): A = J^T J of a row-major m x n Jacobian (FP64),
 * A n x n. KS_FP64: FP64 tiles; KS_MIXED: the 3xTF32 tensor-core GEMM with FP32 accumulation. */
#define KS_TENSOR_TCGEN05 0   /* tcgen05 UMMA, TMA-fed operand tiles, TMEM accumulator (the default) */
#define KS_TENSOR_MMA_SYNC 1  /* mma.sync m16n8k8 (the checked fallback) */

/* Which kernel runs the 3xTF32 GEMMs of the KS_MIXED DFT, its adjoint and ks_normal_matrix (no
 * reference counterpart: the reference's transforms are direct sums). Both read the same split
 * operands and give the same products up to FP32 accumulation order. */
int ks_set_tensor_path(ks_context* ctx, int32_t path);

/* Device time (CUDA events on the context stream) of the 3xTF32 GEMMs since the last reset, their
 * launches and their tensor-core flops (3 x 2 M N K each: the three TF32 products are issued). */
int ks_gemm_stats(ks_context* ctx, double* ms, long long* launches, double* flops, int reset);
int ks_normal_matrix(ks_context* ctx, const double* J, int64_t m, int64_t n, int32_t precision, double* A);

/* sample_adjoint (src/Transfer/transport.jl:221-245) of n independent samples in FP64: for the summed
 * coefficients in (j 4, alpha 4, rho 3 per sample), the step length Dl, the adjoint w in front of the
 * sample and the tail R behind it, out[31 i ..] = O (16, row-major), E (4) and c-bar = (j-bar 4,
 * alpha-bar 4, rho-bar 3), the partials of w^T (O R + E). method 0: the structured form of the mixed
 * path's reverse pass; 1: seven forward-mode duals through the step operator (the reference's form,
 * used by the FP64 adjoint). Arrays host or device. */
int ks_sample_adjoint(ks_context* ctx, int64_t n, const double* in, const double* Dl, const double* w, const double* R, int32_t method,
                      double* out);

/* ---- library extensions with no counterpart in the reference (measurement and streams) ---- */

/* The CUDA stream every call of this context runs on (a cudaStream_t). */
int ks_context_stream(ks_context* ctx, void** stream);

/* Device time (CUDA events on the context stream) of the render kernels since the last reset,
 * their launch count, and the launch count of every kernel of this library. */
int ks_kernel_stats(ks_context* ctx, double* render_ms, long long* render_launches, long long* all_launches, int reset);

/* CUDA graph of one mixed render (the fit loop's forward pass with no host work): records the device
 * work of ks_render(..., KS_MIXED, ...) for device-resident splat sets (params, and hyp of kappa sets,
 * in device memory) and a device `out`: the splat tables built from the parameters, their FP32 copy,
 * the sample stream, the consumer, the segment composition and the output in `order`. The call first
 * renders once the ordinary way (validation, buffers, launch shape). Frames, frequencies, L, nmax,
 * slab, the knot array, the splat counts and all pointers are fixed at capture; every replay re-reads
 * the parameter values, so updating them in place on the device and replaying re-renders. One graph
 * per context; a new capture or ks_graph_destroy releases the previous one. */
int ks_render_graph_capture(ks_context* ctx, const ks_splat_set* sets, int32_t nsets, const double* times, int32_t nframes,
                            const double* nus, int32_t nfreq, double L, int32_t nmax, double slab, double* out, int32_t order);

/* Replay the captured render on the context stream; wait != 0 synchronises (and reports a kernel whose
 * bounded wait gave up, KS_ERR_TIMEOUT). */
int ks_graph_launch(ks_context* ctx, int32_t wait);

/* CUDA graph of one mixed chi^2 + gradient evaluation (chi2_gradient!, Fit.jl:502-534, with chi^2 and
 * its seeds kept on the device as Fit.jl:515-519 would need; no counterpart for the capture itself):
 * records the device work of ks_chi2_gradient(..., KS_MIXED, ...) for device-resident thermal sets and
 * device-resident data, sigma (or the scalar sigma), mask, chi2 (one double) and dparams. That work is
 * the splat and gradient tables from the parameters, the sample stream, the forward pass with the
 * reverse pass's state, chi^2 and its seeds, the reverse pass, the fixed-order reduction into dparams
 * (added when accumulate != 0) and chi^2 into `chi2`. The call first evaluates once the ordinary way,
 * which writes chi2 and dparams. Frames, frequencies, L, nmax, slab, the splat counts and all pointers
 * are fixed at capture; every replay re-reads the parameters and the data. One such graph per context;
 * a new capture releases the previous one, and so do ks_graph_destroy and a new ks_regenerate. */
int ks_chi2_gradient_graph_capture(ks_context* ctx, const ks_splat_set* sets, int32_t nsets, const double* times, int32_t nframes,
                                   const double* nus, int32_t nfreq, double L, int32_t nmax, double slab, const double* data,
                                   const double* sigma, double sigma_scalar, const uint8_t* mask, double* chi2, double* dparams,
                                   int32_t accumulate);

/* Replay the captured chi^2 + gradient evaluation on the context stream; wait != 0 synchronises (and
 * reports a kernel whose bounded wait gave up, KS_ERR_TIMEOUT). */
int ks_chi2_gradient_graph_launch(ks_context* ctx, int32_t wait);

/* Release the captured graphs (the render's and the chi^2 + gradient evaluation's). */
int ks_graph_destroy(ks_context* ctx);

/* Test hook for the bounded waits (no reference counterpart): while on != 0, the mixed kernels arm
 * the shared-memory barrier of their splat-table staging without issuing the copy and poll it only
 * 4096 times, and the tcgen05 GEMM arms its operand barriers without issuing the tile copies and gives
 * each wait ~10 ms, so every block's wait runs out; the kernels record it, free what they hold and
 * return (no fault, no hang) and the call fails with KS_ERR_TIMEOUT. The context stays usable; turn
 * the hook off to render again. */
int ks_set_stage_test(ks_context* ctx, int32_t on);

/* Device time (CUDA events on the context stream) of the persistent consumer k_consume alone in the
 * mixed ks_render calls since the last reset, and its launch count (one per mixed render). */
int ks_consume_stats(ks_context* ctx, double* consume_ms, long long* launches, int reset);

/* Device time (CUDA events) of the adjoint calls (ks_adjoint, ks_chi2_gradient) since the last reset
 * and the launch count of their reverse-pass kernels. */
int ks_adjoint_stats(ks_context* ctx, double* adjoint_ms, long long* launches, int reset);

/* The autotuner of the mixed forward pass: renders the scene (mixed precision) with every block size
 * (384, 256, 128 threads of the persistent consumer, where it fits) and work-unit density (2, 4, 8 or 16
 * work units per resident warp, which sets how finely rays are split into sample segments), `trials`
 * timed renders each after one warm-up, and keeps the fastest for this context's later calls; block,
 * units and best_ms (the render kernels' time) report the choice. */
int ks_autotune(ks_context* ctx, const ks_splat_set* sets, int32_t nsets, const double* times, int32_t nframes, const double* nus,
                int32_t nfreq, double L, int32_t nmax, double slab, int32_t trials, int32_t* block, int32_t* units, double* best_ms);

/* Count work events during ks_render (samples, valid samples, splat tests, weights evaluated,
 * coefficient evaluations, local frames, transfer steps); ks_event_counts reads the 7 counters of
 * the last counted render. */
int ks_set_event_counting(ks_context* ctx, int on);
int ks_event_counts(ks_context* ctx, unsigned long long out[7]);

/* ---- the allocation-free thin image (no counterpart in the reference) ----
 *
 * ks_thin_image_noalloc is ks_thin_image for callers that cannot let a library call cudaMalloc:
 * callers whose device memory is handed out by their own pool (for example a CUDA.jl process, whose
 * allocator must see every byte it owns), and loops where an allocation's implicit device
 * synchronisation would stall the other streams. It allocates nothing: `params` (14 x nsplat,
 * column-major) and `out` (npix doubles, in `order`) must be device pointers the caller owns, the
 * context must have been regenerated (the plan and anchors were allocated then), and the splat table
 * lives in a file-scope device array of KS_NOALLOC_MAX_SPLATS rows (about 100 KB, held by every GPU that
 * loads the library until the process exits). The first call on a device looks up that array's device
 * address (cudaGetSymbolAddress, once per device); make that first call before any stream capture.
 * Every call shares the array: calls that overlap on the GPU race. More than KS_NOALLOC_MAX_SPLATS
 * splats, or host pointers, return KS_ERR_ARGUMENT.
 * Ordering: the call runs on the context stream (ks_context_stream), a non-blocking stream that does
 * not wait for the caller's streams. Whatever writes `params`, or still uses `out`, must be complete
 * before the call: synchronise the stream that does it, or make the context stream wait for it (an
 * event recorded on the caller's stream and cudaStreamWaitEvent on the context stream). Neither
 * allocates. The call is synchronous: it returns after its kernels have finished. */
#define KS_NOALLOC_MAX_SPLATS 256
int ks_thin_image_noalloc(ks_context* ctx, const double* params, int32_t nsplat, double t_obs, int32_t precision,
                          double* out, int32_t order);

#ifdef __cplusplus
}
#endif
#endif /* KERRSPLAT_B200_H */
