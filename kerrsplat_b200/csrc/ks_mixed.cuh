// ks_mixed.cuh -- the mixed-precision transfer consumer with block-cooperative compaction.
//
// k_stream marches every ray once in FP32 (the recurrence and the quadrature, re-anchored to the FP64
// table every M samples) into a sample stream; k_consume walks the stream with one thread per ray
// (sorted slot) in blocks that step through the samples together. What the reference does per sample
// (transport.jl:190-198: every element's coefficients, their sum, one exact step, compositing) is
// spread over the block so that the expensive parts run on full warps (MixedSink):
//   1. every thread with a valid sample tests the candidate splats against the support sphere and
//      the weight cutoff and records the passing (thread, splat) pairs in one block list, in thread
//      order and splat order;
//   2. the block evaluates the listed pairs NT at a time (weight, local frame, synchrotron
//      coefficients at every frequency, cap, invariants, rotation into the screen basis), each thread
//      taking one pair whatever ray it belongs to; the owner then adds the results of its own pairs in
//      splat order (the order of the reference's sum over elements, so the result is deterministic);
//   3. the (thread, frequency) pairs with an active sample are again spread over the block for the
//      exact 4x4 step (O, E), and each owner composes its own steps front to back (S += P E,
//      P = P O; step.jl:347).
// The per-thread Stokes states live in shared memory, the splat table too.
#pragma once
#include "ks_transfer.cuh"

namespace ks {

constexpr float kQCUT = 13.815510557964274f;   // -ln(WEIGHT_CUTOFF): G > 1e-6 <=> q < QCUT

// per-lane sample data (shared memory)
enum SampleField { SF_X, SF_Y, SF_Z, SF_T, SF_PU0, SF_PU1, SF_PU2, SF_PU3, SF_PZ0, SF_PZ1, SF_PZ2, SF_PZ3,
                   SF_LI, SF_OL, SF_SDS, SF_MIS, SF_IVP, SF_R, SF_STH, SF_CTH, SF_SG, SF_ALPHA, SF_BETA, SF_COUNT };
constexpr int kSF = SF_COUNT;                   // floats per lane of sample data
constexpr int kMaxSplatWords = 16;              // candidate masks cover up to 512 splats
constexpr int kGroupWords = 8;                  // candidate words tested before one evaluation list

// The bounds of a work unit's samples (quasi-Cartesian KS box, cylindrical radius and height, and the
// range of their emission times t = t_obs - t~) and the splats whose support can reach them: a
// pattern-rotating splat's support lies within its support radius of the circle its centre runs on
// (rho = ST_RHO, z = ST_CZ), and within it of the arc its centre covers over the unit's emission times
// (the centre's angle is phi_0 + omega (t - t0)); a knot splat's within its bounding sphere (centre
// ST_CX..CZ, radius^2 ST_RHO). Splats outside are below the weight cutoff at every sample of the unit,
// so the per-sample tests skip them (the same result, fewer tests).
struct UnitBox { float xlo, xhi, ylo, yhi, zlo, zhi, rlo, rhi, tlo, thi; };

// Widen the unit box with one sample (position, cylindrical radius, emission time).
__device__ __forceinline__ void unit_box_add(UnitBox& b, float x, float y, float z, float t) {
    const float rho = sqrtf(x * x + y * y);
    b.xlo = fminf(b.xlo, x); b.xhi = fmaxf(b.xhi, x); b.ylo = fminf(b.ylo, y); b.yhi = fmaxf(b.yhi, y);
    b.zlo = fminf(b.zlo, z); b.zhi = fmaxf(b.zhi, z); b.rlo = fminf(b.rlo, rho); b.rhi = fmaxf(b.rhi, rho);
    b.tlo = fminf(b.tlo, t); b.thi = fmaxf(b.thi, t);
}
__device__ __forceinline__ UnitBox unit_box_empty() { return {3e38f, -3e38f, 3e38f, -3e38f, 3e38f, -3e38f, 3e38f, -3e38f, 3e38f, -3e38f}; }

__device__ __forceinline__ float warp_min(float v) {
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, d));
    return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, d));
    return v;
}

// The box of the arc a pattern-rotating splat's centre covers while its rotation angle runs over
// [lo, hi] (relative to the centre's angle at t0), widened by `pad`: the end points and the axis
// extremes the arc passes. False when the arc is not shorter than a turn (then only the circle bounds).
__device__ __forceinline__ bool arc_box(const float* p, float lo, float hi, float pad, float& xlo, float& xhi, float& ylo, float& yhi) {
    if (!(hi - lo < 6.0f)) return false;
    const float rho = p[ST_RHO];
    const float a0 = atan2f(p[ST_CY], p[ST_CX]);
    const float A = a0 + lo, B = a0 + hi;
    float sa, ca, sb, cb;
    sincosf(A, &sa, &ca);
    sincosf(B, &sb, &cb);
    xlo = rho * fminf(ca, cb); xhi = rho * fmaxf(ca, cb); ylo = rho * fminf(sa, sb); yhi = rho * fmaxf(sa, sb);
    // the axis directions 0, pi/2, pi, 3 pi/2 (+ 2 pi k) inside [A, B] (with a margin: conservative)
    const float two_pi = 6.283185307179586f, m = 1e-3f;
    for (int q = 0; q < 4; ++q) {
        const float d = q * 1.5707963267948966f;
        const float k = ceilf((A - m - d) / two_pi);
        if (d + two_pi * k <= B + m) {
            if (q == 0) xhi = rho;
            else if (q == 1) yhi = rho;
            else if (q == 2) xlo = -rho;
            else ylo = -rho;
        }
    }
    xlo -= pad; xhi += pad; ylo -= pad; yhi += pad;
    return true;
}

// The squared radius (about the origin of the quasi-Cartesian frame) beyond which no splat of the
// table can weigh a sample: the pattern rotation keeps a centre's distance from the origin, so a
// pattern-rotating splat reaches |c| + sqrt(support); a knot splat reaches its bounding sphere. Padded
// by 1e-3 relative for the FP32 rounding of the positions. Every thread of the block calls it (the
// table in shared or global memory, values or duals); `slot` is a block-shared float.
template <class TAB>
__device__ __forceinline__ float table_reach2(const TAB* tab, int ntot, float* slot) {
    if (threadIdx.x == 0) *slot = 0.f;
    __syncthreads();
    float m = 0.f;
    for (int i = threadIdx.x; i < ntot; i += blockDim.x) {
        const TAB* p = tab + (long long)i * ST_COUNT;
        const float cx = float(value_of(p[ST_CX])), cy = float(value_of(p[ST_CY])), cz = float(value_of(p[ST_CZ]));
        const bool knot = int(value_of(p[ST_KIND])) == KS_KNOT21;
        const float c = sqrtf(cx * cx + cy * cy + cz * cz);
        m = fmaxf(m, c + sqrtf(float(value_of(knot ? p[ST_RHO] : p[ST_SUPP]))));
    }
    atomicMax(reinterpret_cast<int*>(slot), __float_as_int(m));   // non-negative floats order as ints
    __syncthreads();
    const float r = *slot * 1.001f + 1e-3f;
    return r * r;
}

// the candidate mask words of a unit (all lanes call it; cand gets ceil(ntot / 32) words)
__device__ __forceinline__ void unit_candidates(const float* tab, int ntot, const UnitBox& b, int lane, unsigned* cand) {
    for (int s0 = 0; s0 < ntot; s0 += 32) {
        const int i = s0 + lane;
        bool keep = false;
        if (i < ntot && b.xlo <= b.xhi) {
            const float* p = tab + i * ST_COUNT;
            if (int(p[ST_KIND]) == KS_KNOT21) {
                const float dx = fmaxf(fmaxf(b.xlo - p[ST_CX], p[ST_CX] - b.xhi), 0.f);
                const float dy = fmaxf(fmaxf(b.ylo - p[ST_CY], p[ST_CY] - b.yhi), 0.f);
                const float dz = fmaxf(fmaxf(b.zlo - p[ST_CZ], p[ST_CZ] - b.zhi), 0.f);
                keep = dx * dx + dy * dy + dz * dz <= p[ST_RHO] * 1.0001f;
            } else {
                const float dr = fmaxf(fmaxf(b.rlo - p[ST_RHO], p[ST_RHO] - b.rhi), 0.f);
                const float dz = fmaxf(fmaxf(b.zlo - p[ST_CZ], p[ST_CZ] - b.zhi), 0.f);
                keep = dr * dr + dz * dz <= p[ST_SUPP] * 1.0001f;
                float xlo, xhi, ylo, yhi;
                const float om = p[ST_OMEGA];
                const float pa = om * (b.tlo - p[ST_T0]), pb = om * (b.thi - p[ST_T0]);
                // the pad covers the FP32 rounding of the angles (phases up to ~1e3 rad) and positions
                const float pad = 1e-3f * p[ST_RHO] + 1e-4f * (fabsf(pa) + fabsf(pb)) * p[ST_RHO] + 1e-3f;
                if (keep && b.tlo <= b.thi && arc_box(p, fminf(pa, pb), fmaxf(pa, pb), pad, xlo, xhi, ylo, yhi)) {
                    const float dx = fmaxf(fmaxf(b.xlo - xhi, xlo - b.xhi), 0.f);
                    const float dy = fmaxf(fmaxf(b.ylo - yhi, ylo - b.yhi), 0.f);
                    keep = dx * dx + dy * dy + dz * dz <= p[ST_SUPP] * 1.0001f;
                }
            }
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (lane == 0) cand[s0 >> 5] = m;
    }
    __syncwarp();
}

// The warp's union of its lanes' boxes.
__device__ __forceinline__ void unit_box_reduce(UnitBox& b) {
    b.xlo = warp_min(b.xlo); b.xhi = warp_max(b.xhi); b.ylo = warp_min(b.ylo); b.yhi = warp_max(b.yhi);
    b.zlo = warp_min(b.zlo); b.zhi = warp_max(b.zhi); b.rlo = warp_min(b.rlo); b.rhi = warp_max(b.rhi);
    b.tlo = warp_min(b.tlo); b.thi = warp_max(b.thi);
}

// ---- TMA bulk staging ----------------------------------------------------------------------------

constexpr int kStageWaitLimit = 1 << 22;   // mbarrier polls before a staging copy is declared lost

__device__ __forceinline__ unsigned smem_u32(const void* p) { return unsigned(__cvta_generic_to_shared(p)); }

// Stage `bytes` (a multiple of 16; both addresses 16-byte aligned) from global memory into this CTA's
// shared memory with one TMA bulk copy (cp.async.bulk, no multicast) completing on the mbarrier `bar`.
// Every thread of the block calls it; thread 0 initialises the barrier and issues the copy, all
// threads wait for the barrier's phase 0 with a bounded number of polls. Returns false (the same in
// every thread) when the copy did not land within the limit: the caller records an error and returns.
// With issue == false (a test of the error path) the barrier is armed but no copy is issued, so every
// thread's wait runs out after `limit` polls and the function returns false.
__device__ __forceinline__ bool stage_bulk(void* dst, const void* src, unsigned bytes, unsigned long long* bar, bool issue = true,
                                           int limit = kStageWaitLimit) {
    const unsigned b = smem_u32(bar);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared.b64 [%0], 1;" ::"r"(b) : "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // the barrier, visible to the copy engine
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared.b64 st, [%0], %1;\n\t}" ::"r"(b), "r"(bytes) : "memory");
        if (issue)
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                         ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(b) : "memory");
    }
    unsigned done = 0;
    for (int it = 0; it < limit && !done; ++it)
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared.b64 p, [%1], 0;\n\tselp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done) : "r"(b) : "memory");
    return __syncthreads_and(done != 0) != 0;
}

// Exclusive scan of v over the NT threads of a block, total = the block sum. One barrier: the warp
// sums alternate between the two halves of ws2 ([2][NT / 32], `par` toggles on every call, the same
// sequence in every thread), so a scan never overwrites sums a slower warp of the previous scan is
// still reading.
template <int NT>
__device__ __forceinline__ int block_exscan(int v, int& total, int* ws2, int& par) {
    constexpr int W = NT / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int* ws = ws2 + par * W;
    par ^= 1;
    int incl = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += u;
    }
    if (lane == 31) ws[warp] = incl;
    __syncthreads();
    int pre = 0, tot = 0;
#pragma unroll
    for (int q = 0; q < W; ++q) {
        const int sv = ws[q];
        pre += (q < warp) ? sv : 0;
        tot += sv;
    }
    total = tot;
    return pre + incl - v;
}

template <int CH>
struct MixedSmem {
    // per-warp shares of the block's regions (the splat table comes first); the block pools them:
    // sample data [kSF][NT], pair list | step results, pair results [CH * 12][NT], meta, states
    static constexpr int kSampleBytes = 32 * kSF * 4;
    static constexpr int kItemBytes = 32 * 20 * 4;                                              // pair list (4 B items) | step results [20][NT]
    static constexpr int kResBytes = 32 * CH * 12 * 4;                                          // pair results | step inputs | pass masks
    static constexpr int kMetaBytes = 32 * 4 * 2 + kMaxSplatWords * 4 + 2 * 4 + 4 * 4;           // step offsets, bits; candidate mask; scan sums; class counts
    static constexpr int kStateBytes = 32 * CH * 20 * 4;                                        // P (16) and S (4) per thread and frequency
    static constexpr int kWarpBytes = kSampleBytes + kItemBytes + kResBytes + kMetaBytes + kStateBytes;
    static_assert(kGroupWords * 32 * 4 <= kResBytes, "a group's pass masks fit in the pair-results buffer");
    static_assert(32 * kMaxSplatWords <= 512, "items carry 9-bit splat indices");
    // the splat table and the knot array (nkv floats) come first
    __host__ __device__ static size_t tab_bytes(int ntot, int nkv) { return (size_t(ntot) * ST_COUNT * 4 + size_t(nkv) * 4 + 15) / 16 * 16; }
    static size_t bytes(int ntot, int warps, int nkv = 0) { return tab_bytes(ntot, nkv) + size_t(warps) * kWarpBytes; }
};

// Out-of-line pieces of the consumer: one copy of each in the instruction cache (inlined into the
// per-frequency loop and the three populations they overflowed it; ncu: "no instruction" stalls).
// s: the owner's column of the block's sample data ([field][NT] layout)
template <int NT>
__device__ __noinline__ LFrame<float> local_frame_ool(const float* s, const float* p, float a, float a_sin_tho) {
    SampleFrame<float> F;
    F.pu[0] = s[SF_PU0 * NT]; F.pu[1] = s[SF_PU1 * NT]; F.pu[2] = s[SF_PU2 * NT]; F.pu[3] = s[SF_PU3 * NT];
    F.pz[0] = s[SF_PZ0 * NT]; F.pz[1] = s[SF_PZ1 * NT]; F.pz[2] = s[SF_PZ2 * NT]; F.pz[3] = s[SF_PZ3 * NT];
    F.lapse_inv = s[SF_LI * NT]; F.om_lapse = s[SF_OL * NT]; F.sDS = s[SF_SDS * NT]; F.misS = s[SF_MIS * NT]; F.ivarpi = s[SF_IVP * NT];
    F.r = s[SF_R * NT]; F.sth = s[SF_STH * NT]; F.cth = s[SF_CTH * NT]; F.a = a;
    return local_frame(F, p[ST_U1], p[ST_U2], p[ST_U3], p[ST_BHX], p[ST_BHY], p[ST_BHZ], p[ST_BZERO] != 0.f,
                       s[SF_ALPHA * NT], s[SF_BETA * NT], a_sin_tho);
}

// Screen-basis coefficients of one splat at one frequency (transport.jl:265-270), written with a
// stride of NT floats: j (4), alpha (4), rho (3), active flag.
// KM: the populations the scene contains (bit 0 thermal, 1 power law, 2 kappa); the kernel for a
// thermal-only scene carries none of the other fits' code.
template <int KM, int NT>
__device__ __noinline__ void screen_coefficients_ool(int kind, const float* p, float ne, float nuf, float sb, float cb, float s2c, float c2c,
                                                     float* r) {
    Coef<float> cf;
    if ((KM & 2) && kind == KS_POWERLAW22)
        cf = powerlaw_cs(ne, p[ST_P], p[ST_GMIN], p[ST_GSPAN], p[ST_GAMJ], p[ST_GAMA], p[ST_BMAG], nuf, sb, cb);
    else if ((KM & 4) && kind == KS_KAPPA22)
        cf = kappa_cs(ne, p[ST_KAP], p[ST_W], p[ST_HYP], p[ST_G43], p[ST_G2], p[ST_GQ], p[ST_GP], p[ST_GK2], p[ST_KB], p[ST_BMAG], nuf, sb, cb);
    else
        cf = thermal_cs(ne, p[ST_TE], p[ST_F0], p[ST_KR], p[ST_BMAG], nuf, sb, cb);
    bool on = cf.jI > 0.f || cf.aI > 0.f || cf.rQ != 0.f || cf.rV != 0.f;
    if (!on) { r[11 * NT] = 0.f; return; }
    float fe = cap_factor(cf.jI, cf.jQ, cf.jV, 0.99f);
    float fa = cap_factor(cf.aI, cf.aQ, cf.aV, 0.99f);
    float nh = nuf / float(kNU0);
    float i2 = 1.f / (nh * nh);
    float jQ = cf.jQ * fe * i2, aQ = cf.aQ * fa * nh, rQ = cf.rQ * nh;
    r[0] = cf.jI * i2; r[NT] = jQ * c2c; r[2 * NT] = jQ * s2c; r[3 * NT] = cf.jV * fe * i2;
    r[4 * NT] = nh * cf.aI; r[5 * NT] = aQ * c2c; r[6 * NT] = aQ * s2c; r[7 * NT] = cf.aV * fa * nh;
    r[8 * NT] = rQ * c2c; r[9 * NT] = rQ * s2c; r[10 * NT] = nh * cf.rV;
    r[11 * NT] = 1.f;
}

// The exact step of one (owner, frequency): reads the owner's summed coefficients from shared memory
// (11 values NT apart) and writes O (16) and E (4) to shared memory (NT apart): no arrays cross the
// call (passed through the stack they cost a local store per element, most of them L1 misses).
template <int NT>
__device__ __noinline__ void transfer_step_ool(const float* in, float Dl, float* out) {
    float v[11];
#pragma unroll
    for (int q = 0; q < 11; ++q) v[q] = in[q * NT];
    float o[16], e[4];
    transfer_step_structured(c_moments, v, v + 4, v + 8, Dl, o, e);
#pragma unroll
    for (int q = 0; q < 16; ++q) out[q * NT] = o[q];
#pragma unroll
    for (int q = 0; q < 4; ++q) out[(16 + q) * NT] = e[q];
}

// The consumer of one thread (one ray) of a block work unit: all NT threads of the block call
// consume() for the same sample together. What the reference does per sample (transport.jl:190-198:
// every element's coefficients, their sum, one exact step, compositing) is spread over the block:
//   1. every thread with a valid sample tests the unit's candidate splats against the support and
//      the weight cutoff, and the passing (thread, splat) pairs of up to kGroupWords candidate words
//      go into one block list (thread order, splat order within a thread);
//   2. the block evaluates the list NT pairs at a time (weight, local frame, synchrotron
//      coefficients at every frequency, cap, invariants, rotation into the screen basis), each thread
//      taking one pair whatever ray it belongs to, and every owner adds the results of its own pairs
//      in list order (the reference's order of the sum over elements: deterministic);
//   3. the (thread, frequency) pairs with an active sample are spread over the block for the exact
//      4x4 step (O, E), and each owner composes its steps front to back (S += P E, P = P O;
//      step.jl:347).
// Block lists keep every round full across warps: with per-warp lists the warps of a block waited at
// the phase barriers for the one with the most pairs.
template <int CH, int KM, int NT>
struct MixedSink {
    static constexpr int W = NT / 32;
    static_assert(NT <= 512, "items carry 9-bit owner indices");
    const float* tab; int ntot;
    const float* knots;   // the knot array of knot splats (after the table)
    float t_obs;
    float nu[CH], Lnu[CH];
    int nc;
    float a, rh_lo, dtau, alpha, beta, eta, lam, a_sin_tho, slab;
    float reach2;     // table_reach2: samples farther out test no splat
    int nmax;
    int tid;
    bool live;        // false for the padding threads past the last ray
    float* sf;        // the block's sample data [kSF][NT]
    unsigned* items;  // the block's pair list (item_cap entries: owner << 9 | splat)
    float* sres;      // step results [20][NT] (aliases the pair list)
    float* res;       // pair results [CH * 12][NT] | step inputs | a group's pass masks [kGroupWords][NT]
    float* state;     // this thread's P/S column of the block's [CH * 20][NT] array
    int* meta_off;    // the block's first step item per thread [NT]
    unsigned* meta_bits;   // and active-frequency bits [NT]
    int* wsum;        // warp sums of the block scans, double-buffered [2][W]
    int scan_par;
    int item_cap;
    bool sort_kinds;       // the scene mixes populations or has knot splats: evaluate each round grouped by class
    int* kcnt;             // per-warp class counts of a round [W][4]
    const unsigned* cand;  // this warp's candidate splats (unit_candidates)
    float zprev; int wn; bool inside, crossed, zset;
    unsigned int ev[7];
    // the adjoint's forward pass (null otherwise): at every active (sample, thread, frequency) the
    // state P before the sample (16) and the summed coefficients (11) into gstate[((combo N + k - 1)
    // 27 + field) npad + ray], and gact[(combo N + k - 1) npad + ray] = 1; jbase = the block's first ray
    float* gstate;
    unsigned char* gact;
    long long gnpad, jbase;
    int gN, kcur, gframes, gf, gv0;
    int nsamp;        // this thread's samples

    __device__ void init() {
        for (int c = 0; c < CH; ++c) {
            float* st = state + c * 20 * NT;
            for (int q = 0; q < 16; ++q) st[q * NT] = (q % 5 == 0) ? 1.f : 0.f;
            for (int q = 16; q < 20; ++q) st[q * NT] = 0.f;
        }
        for (int q = 0; q < 7; ++q) ev[q] = 0;
        wn = 0; inside = false; crossed = false; zset = false; zprev = 0.f;
    }

    __device__ bool wind_ok(float z) {   // step.jl:379-398; returns whether the sample is kept
        if (!zset) { zprev = z; zset = true; inside = fabsf(z) < slab; crossed = false; return wn <= nmax; }
        bool inside_now = fabsf(z) < slab;
        bool crossing = zprev * z < 0.f;
        if (inside || inside_now) {
            crossed = crossed || crossing;
            if (inside && !inside_now) { if (crossed) wn += 1; crossed = false; }
            else if (!inside && inside_now) { crossed = crossing; }
            inside = inside_now;
        } else if (crossing) {
            wn += 1;
        }
        zprev = z;
        return wn <= nmax;
    }

    __device__ int scan(int v, int& total) { return block_exscan<NT>(v, total, wsum, scan_par); }


    // The evaluation class of a pair: 0 thermal, 1 knot (thermal coefficients, knot centre), 2 power
    // law, 3 kappa; 4 for a thread without a pair this round.
    __device__ int pair_class(int kk, int wt) const {
        if (kk >= wt) return 4;
        const int kind = int(tab[int(items[kk] & 511u) * ST_COUNT + ST_KIND]);
        return kind == KS_KNOT21 ? 1 : kind == KS_POWERLAW22 ? 2 : kind == KS_KAPPA22 ? 3 : 0;
    }

    // The round's pairs [base, base + NT) of the list re-dealt to the threads grouped by class (a
    // counting sort over warp ballots; two barriers), so that a warp runs one population's fit instead
    // of all of them in turn. The results still go to each pair's own slot, so the owners' sums keep
    // list order. Returns the list index this thread evaluates (>= wt: none).
    __device__ int kind_sorted(int kk0, int wt, int base) {
        const int lane = tid & 31, warp = tid >> 5;
        const int cls = pair_class(kk0, wt);
        unsigned mine = 0u;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const unsigned m = __ballot_sync(0xffffffffu, cls == k);
            if (lane == 0) kcnt[warp * 4 + k] = __popc(m);
            if (cls == k) mine = m;
        }
        __syncthreads();
        int dst = NT;   // no pair: nothing to place
        if (cls < 4) {
            dst = __popc(mine & ((1u << lane) - 1u));
            for (int w = 0; w < W; ++w)
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    dst += (k < cls || (k == cls && w < warp)) ? kcnt[w * 4 + k] : 0;
            meta_off[dst] = kk0;   // the step offsets are free during the evaluations
        }
        __syncthreads();
        return (tid < min(NT, wt - base)) ? meta_off[tid] : wt;
    }

    // pair (owner o, splat i): weight, frame, coefficients at every frequency -> res slot
    __device__ void evaluate(int o, int i, float* out) {
        // the block's sample data is stored field-major ([field][thread]) so that threads hit distinct banks
        const float* s = sf + o;
        const float* p = tab + i * ST_COUNT;
        const int kind = int(p[ST_KIND]);
        float q;
        if (kind == KS_KNOT21) knot_exponent(p, knots, t_obs - s[SF_T * NT], s[SF_X * NT], s[SF_Y * NT], s[SF_Z * NT], q);
        else splat_exponent(p, t_obs - s[SF_T * NT], s[SF_X * NT], s[SF_Y * NT], s[SF_Z * NT], false, q);
        float G = __expf(-q);
        LFrame<float> lf = local_frame_ool<NT>(s, p, a, a_sin_tho);
        float sb, cb;
        pitch_sc(lf.cosB, sb, cb);
        float ne = p[ST_NE] * G;
        const float s2c = lf.s2c, c2c = lf.c2c;
#pragma unroll 1
        for (int c = 0; c < CH; ++c) {
            float* r = out + c * 12 * NT;   // out = res + slot; fields are NT apart
            if (c >= nc) { r[11 * NT] = 0.f; continue; }
            float nuc = nu[0];
#pragma unroll
            for (int cc = 1; cc < CH; ++cc) nuc = (cc == c) ? nu[cc] : nuc;
            screen_coefficients_ool<KM, NT>(kind, p, ne, nuc / lf.g, sb, cb, s2c, c2c, r);
        }
        // the work events of the pair, counted as the FP64 consumer counts them: one local frame
        // (shared by the frequencies) and one coefficient evaluation per frequency
        ev[4] += nc;
        ev[5] += 1;
    }

    // The consumer for one sample of every thread of the block (all NT threads call it together):
    // `usable` = Krang's validity and outside r_h (1 + 1e-3) (transport.jl:171-173); x, y, z the
    // quasi-Cartesian Kerr-Schild position, ts the regularized lookback time t~.
    __device__ void consume(bool usable, float x, float y, float z, float ts, float r, float sth, float cth, bool nur, bool nuth) {
        const bool inrange = kcur <= nsamp;   // a ray with fewer samples than the unit's segment
        if (inrange) ev[0]++;
        bool valid = live && inrange && usable;
        if (valid) ev[1]++;
        if (valid && nmax >= 0) valid = wind_ok(r * cth);
        // beyond every splat's reach a sample has no pair: its tests are skipped (they would all fail)
        const bool testable = valid && x * x + y * y + z * z <= reach2;
        float* mys = sf + tid;
        float t = 0.f, rho = 0.f;
        if (valid) {
            rho = sqrtf(x * x + y * y);
            t = t_obs - ts;
            mys[SF_X * NT] = x; mys[SF_Y * NT] = y; mys[SF_Z * NT] = z; mys[SF_T * NT] = ts;
        }
        bool framed = false;   // the sample's frame data is formed at its first passing pair
        float acc[CH][11];
        unsigned actbits = 0u;
#pragma unroll
        for (int c = 0; c < CH; ++c)
#pragma unroll
            for (int q = 0; q < 11; ++q) acc[c][q] = 0.f;
        // Tests over groups of up to kGroupWords candidate words (256 splats), one block list per
        // group. The group's pass masks are kept in the pair-results buffer until the list is written
        // (it is free until the evaluations). A group whose list would overflow is redone one chunk
        // (32 splats, the mask in a register) at a time, in windows of item_cap pairs.
        const int nw = (ntot + 31) >> 5;
        unsigned* gmask = reinterpret_cast<unsigned*>(res) + tid;   // [kGroupWords][NT]
        int single_end = -1;   // chunks below this index go one at a time
        for (int g0 = 0; g0 < nw;) {
            const bool single = g0 < single_end;
            const int g1 = single ? g0 + 1 : min(nw, g0 + kGroupWords);
            int n = 0;
            unsigned m1 = 0u;
            for (int wd = g0; wd < g1; ++wd) {
                const unsigned cm = cand[wd];
                unsigned mask = 0u;
                if (testable && cm) {
                    unsigned cbits = cm;
                    while (cbits) {
                        const int b = __ffs(cbits) - 1;
                        cbits &= cbits - 1;
                        const float* p = tab + (wd * 32 + b) * ST_COUNT;
                        float q;
                        ev[2]++;
                        // the pattern rotation keeps the centre on a circle about the spin axis: a point
                        // farther than the support radius from that circle is outside the support sphere
                        // at every time (no trigonometry needed)
                        const float dr = rho - p[ST_RHO], dz = z - p[ST_CZ];
                        if (int(p[ST_KIND]) != KS_KNOT21) {
                            if (dr * dr + dz * dz > p[ST_SUPP]) continue;
                            if (!splat_exponent(p, t, x, y, z, true, q)) continue;
                        } else {
                            const float dx = x - p[ST_CX], dy = y - p[ST_CY], dz2 = z - p[ST_CZ];
                            if (dx * dx + dy * dy + dz2 * dz2 > p[ST_RHO]) continue;   // outside the knots' bounding sphere
                            knot_exponent(p, knots, t, x, y, z, q);
                        }
                        ev[3]++;
                        if (q < kQCUT) mask |= 1u << b;
                    }
                }
                if (single) m1 = mask;
                else gmask[(wd - g0) * NT] = mask;
                n += __popc(mask);
            }
            int total;
            const int off = scan(n, total);   // block-uniform total: every thread takes the same branches
            if (!single && total > item_cap) { single_end = g1; continue; }
            if (n > 0 && !framed) {
                // what the evaluations of this thread's pairs read: the sample's frame, position, Sigma dtau
                const SampleFrame<float> F = sample_frame(a, r, 0.f, sth, cth, eta, lam, nur, nuth);
                mys[SF_PU0 * NT] = F.pu[0]; mys[SF_PU1 * NT] = F.pu[1]; mys[SF_PU2 * NT] = F.pu[2]; mys[SF_PU3 * NT] = F.pu[3];
                mys[SF_PZ0 * NT] = F.pz[0]; mys[SF_PZ1 * NT] = F.pz[1]; mys[SF_PZ2 * NT] = F.pz[2]; mys[SF_PZ3 * NT] = F.pz[3];
                mys[SF_LI * NT] = F.lapse_inv; mys[SF_OL * NT] = F.om_lapse; mys[SF_SDS * NT] = F.sDS; mys[SF_MIS * NT] = F.misS;
                mys[SF_IVP * NT] = F.ivarpi;
                mys[SF_R * NT] = r; mys[SF_STH * NT] = sth; mys[SF_CTH * NT] = cth;
                mys[SF_SG * NT] = (r * r + a * a * cth * cth) * dtau;   // Sigma dtau of this thread's ray
                mys[SF_ALPHA * NT] = alpha; mys[SF_BETA * NT] = beta;
                framed = true;
            }
            for (int wb = 0; wb < total; wb += item_cap) {
                // this thread's pairs with list index in [wb, wb + item_cap)
                if (n > 0 && off + n > wb && off < wb + item_cap) {
                    int k = off;
                    for (int wd = g0; wd < g1; ++wd) {
                        unsigned m = single ? m1 : gmask[(wd - g0) * NT];
                        while (m) {
                            const int b = __ffs(m) - 1;
                            m &= m - 1;
                            if (k >= wb && k < wb + item_cap) items[k - wb] = (unsigned(tid) << 9) | unsigned(wd * 32 + b);
                            ++k;
                        }
                    }
                }
                __syncthreads();
                // 2. evaluation rounds over the block, then owner accumulation in list order
                const int wt = min(item_cap, total - wb);
                for (int base = 0; base < wt; base += NT) {
                    int kk0 = base + tid;
                    if (sort_kinds) kk0 = kind_sorted(kk0, wt, base);
                    if (kk0 < wt) {
                        const unsigned it = items[kk0];
                        evaluate(int(it >> 9), int(it & 511u), res + (kk0 - base));
                    }
                    __syncthreads();
                    const int lo = max(off, wb + base), hi = min(off + n, wb + base + NT);
                    for (int kk = lo; kk < hi; ++kk) {
                        const float* rr = res + (kk - wb - base);
#pragma unroll
                        for (int c = 0; c < CH; ++c) {
                            if (rr[(c * 12 + 11) * NT] != 0.f) {
#pragma unroll
                                for (int q = 0; q < 11; ++q) acc[c][q] += rr[(c * 12 + q) * NT];
                                actbits |= 1u << c;
                            }
                        }
                    }
                    __syncthreads();
                }
            }
            g0 = g1;
        }
        // 3. steps: (thread, frequency) pairs with active coefficients, spread over the block
        const int n2 = __popc(actbits);
        int total2;
        const int off2 = scan(n2, total2);
        if (total2 == 0) return;
        // publish this thread's sums (step inputs) in the results buffer: [c][12][NT]
#pragma unroll
        for (int c = 0; c < CH; ++c)
#pragma unroll
            for (int q = 0; q < 11; ++q) res[(c * 12 + q) * NT + tid] = acc[c][q];
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
                // its (g - off)-th active frequency
                unsigned bits = meta_bits[o];
                const int j = g - meta_off[o];
                for (int q = 0; q < j; ++q) bits &= bits - 1;
                const int c = __ffs(bits) - 1;
                const float* in = res + (c * 12) * NT + o;   // the owner's sums, NT apart
                float Lc = Lnu[0];
#pragma unroll
                for (int cc = 1; cc < CH; ++cc) Lc = (cc == c) ? Lnu[cc] : Lc;   // no dynamic register indexing
                const float Dl = Lc * sf[SF_SG * NT + o];   // the owner's Sigma dtau
                transfer_step_ool<NT>(in, Dl, sres + tid);
                if (gstate) {
                    const long long combo = (long long)(gv0 + c) * gframes + gf;
                    float* gs = gstate + ((combo * gN + (kcur - 1)) * 27 + 16) * gnpad + jbase + o;
#pragma unroll
                    for (int q = 0; q < 11; ++q) gs[q * gnpad] = in[q * NT];
                }
            }
            __syncthreads();
            // owners compose their steps front to back (frequency order)
            const int lo = max(off2, base), hi = min(off2 + n2, base + NT);
            if (lo < hi) {
                unsigned bits = actbits;
                for (int q = off2; q < lo; ++q) bits &= bits - 1;
                for (int g2 = lo; g2 < hi; ++g2) {
                    const int c = __ffs(bits) - 1;
                    bits &= bits - 1;
                    float OE[20];
#pragma unroll
                    for (int q = 0; q < 20; ++q) OE[q] = sres[q * NT + (g2 - base)];
                    float* st = state + c * 20 * NT;   // this thread's column, fields NT apart
                    float P[16], S4[4];
#pragma unroll
                    for (int q = 0; q < 16; ++q) P[q] = st[q * NT];
                    if (gstate) {
                        const long long combo = (long long)(gv0 + c) * gframes + gf;
                        const long long row = combo * gN + (kcur - 1);
                        float* gs = gstate + row * 27 * gnpad + jbase + tid;
#pragma unroll
                        for (int q = 0; q < 16; ++q) gs[q * gnpad] = P[q];
                        gact[row * gnpad + jbase + tid] = 1;
                    }
#pragma unroll
                    for (int q = 0; q < 4; ++q) S4[q] = st[(16 + q) * NT];
#pragma unroll
                    for (int r4 = 0; r4 < 4; ++r4) {
                        S4[r4] += P[4 * r4] * OE[16] + P[4 * r4 + 1] * OE[17] + P[4 * r4 + 2] * OE[18] + P[4 * r4 + 3] * OE[19];
#pragma unroll
                        for (int q = 0; q < 4; ++q)
                            st[(4 * r4 + q) * NT] = P[4 * r4] * OE[q] + P[4 * r4 + 1] * OE[4 + q] + P[4 * r4 + 2] * OE[8 + q] + P[4 * r4 + 3] * OE[12 + q];
                    }
#pragma unroll
                    for (int q = 0; q < 4; ++q) st[(16 + q) * NT] = S4[q];
                    ev[6]++;
                }
            }
            __syncthreads();
        }
    }
};

// ks_coords is defined in ks_lib.cu before this header is included.

// The FP32 sample stream: every sample of every ray, marched once per render (the recurrence and the
// quadrature re-anchored to the FP64 table) and shared by every frame, frequency and parameter set.
// Layout [k][field][npad] (k = sample - 1): the lanes of a warp (consecutive sorted rays) read and
// write consecutive addresses.
enum StreamField { SM_X, SM_Y, SM_Z, SM_T, SM_R, SM_STH, SM_CTH, SM_FLAGS, SM_COUNT };

// T: the precision of the march (float: the mixed path; double: FP64 geodesics with the transport in
// FP32, the reference's `precision(cache, Float32)` arrangement, cache.jl:212-232). The stream is FP32.
template <class T>
struct StreamSink {
    float* out;
    long long npad, j;
    T a, rh_lo;
    T rp, rm;       // the horizons
    float afac;     // a / (2 sqrt(1 - a^2))
    // The quasi-Cartesian Kerr-Schild position of ks_coords in the precision of the stream: the sample
    // is FP64 (T = double) but x, y, z are stored in FP32, so the angles go to FP32 trigonometry once
    // phi_KS is reduced into [-pi, pi] in T; sin theta comes from cos theta (sqrt((1 - c)(1 + c)),
    // as accurate as sin(acos c)); r - r_+ and r - r_- are formed in T before the FP32 logarithm.
    __device__ void operator()(int k, const Sample<T>& s) {
        float* o = out + (long long)(k - 1) * SM_COUNT * npad + j;
        const bool usable = s.ok && s.r > rh_lo;
        unsigned flags = (s.ok ? 1u : 0u) | (s.nur ? 2u : 0u) | (s.nutheta ? 4u : 0u) | (usable ? 8u : 0u);
        float x = 0.f, y = 0.f, z = 0.f, sth = 0.f, cth = 0.f;
        if (usable) {
            const T c = s.cos_theta;
            const T st2 = (T(1) - c) * (T(1) + c);
            cth = float(c);
            sth = float(sqrt(st2 > T(0) ? st2 : T(0)));
            const float lg = logf(fabsf(float(s.r - rp + keps<T>()) / float(s.r - rm + keps<T>())));
            const T phks = s.phi + T(afac * lg - atan2f(float(a), float(s.r)));
            const T turns = rint(phks * T(0.15915494309189535));   // 1 / (2 pi)
            const float phr = float(phks - turns * T(6.283185307179586));
            float sp, cp;
            sincosf(phr, &sp, &cp);
            const float r = float(s.r);
            x = r * sth * cp; y = r * sth * sp; z = r * cth;
        }
        o[SM_X * npad] = x; o[SM_Y * npad] = y; o[SM_Z * npad] = z; o[SM_T * npad] = float(s.t);
        o[SM_R * npad] = float(s.r); o[SM_STH * npad] = sth; o[SM_CTH * npad] = cth;
        o[SM_FLAGS * npad] = __uint_as_float(flags);
    }
};

// One thread per (ray, segment of seg_len samples starting at an anchor multiple). At most 128
// registers (four blocks per SM): the FP64 march held 252 and ran 8 warps per SM; capped, 16 warps
// per SM hide more of the FP64 latency (4% of the configuration-2 render, same stream).
template <class T>
__global__ void __launch_bounds__(128, 4) k_stream(PlanView P, Spacetime st, long long npix, int seg_len, int nseg, float* __restrict__ out) {
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= npix * nseg) return;
    const long long j = q % npix;
    const int seg = int(q / npix);
    const int k0 = 1 + seg * seg_len, k1 = min(st.N + 1, k0 + seg_len);
    MarchRay<T> R = load_ray<T>(P, st, j);
    const double temp = sqrt(1.0 - st.a * st.a);
    StreamSink<T> sink{out, P.npad, j, T(st.a), T(st.rh * (1 + 1e-3)), T(1.0 + temp), T(1.0 - temp), float(st.a / (2.0 * temp))};
    march_range(P, j, R, sink, k0, k1);
}

// Persistent consumer: every warp takes work units (32 consecutive sorted rays x one segment of the
// sample range x one frame and up to CH frequencies) from a device counter until none is left, the
// last rays first (the plunging rays near the centre of the screen, sorted last, carry most of the
// transport work). A segment [k0, k1) composes its own (P, S) from the identity; k_combine
// composes the segments of a ray front to back (S = S_0 + P_0 (S_1 + P_1 (...))).
struct MixedJob {
    long long npix, npad;
    int nframes, nfreq, nseg, seg_len, nvc;
    long long nchunks, total;
    int nmax;
    float slab;
    double L;
    float* gstate = nullptr;          // the adjoint's per-sample states (see MixedSink)
    unsigned char* gact = nullptr;
    int nkv = 0;                      // knot values after the splat table
    int ch = 1;                       // frequencies per work unit
    int cand_len = 0;                 // samples per candidate mask (0: the whole segment)
    int stage_test = 0;               // test hook: arm the table-staging barrier without the copy
};

template <int CH, int NT, int KM>
__global__ void __launch_bounds__(NT, 1)
k_consume(PlanView P, Spacetime st, MixedJob job, const float* __restrict__ tab32, int ntot, const double* __restrict__ ct,
          const double* __restrict__ cnu, const float* __restrict__ stream, unsigned long long* __restrict__ work,
          float* __restrict__ seg_out, unsigned long long* __restrict__ counters, unsigned* __restrict__ err) {
    extern __shared__ __align__(16) unsigned char smem[];
    float* tab = reinterpret_cast<float*>(smem);
    // the FP32 splat table and knot array (padded to 16 bytes) into shared memory by one bulk copy
    __shared__ __align__(8) unsigned long long tab_bar;
    const unsigned tab_bytes = unsigned(MixedSmem<CH>::tab_bytes(ntot, job.nkv));
    if (tab_bytes > 0 && !stage_bulk(tab, tab32, tab_bytes, &tab_bar, job.stage_test == 0, job.stage_test ? 4096 : kStageWaitLimit)) {
        if (threadIdx.x == 0) atomicOr(err, 1u);
        return;
    }
    // the block's regions after the table (each the sum of the warps' shares, MixedSmem)
    using MS = MixedSmem<CH>;
    constexpr int W = NT / 32;
    unsigned char* bb = smem + MS::tab_bytes(ntot, job.nkv);
    float* sf_b = reinterpret_cast<float*>(bb);
    unsigned char* items_b = bb + W * MS::kSampleBytes;
    float* res_b = reinterpret_cast<float*>(items_b + W * MS::kItemBytes);
    int* meta_off_b = reinterpret_cast<int*>(reinterpret_cast<unsigned char*>(res_b) + W * MS::kResBytes);
    unsigned* meta_bits_b = reinterpret_cast<unsigned*>(meta_off_b + NT);
    unsigned* cand_b = meta_bits_b + NT;                                   // [W][kMaxSplatWords]
    int* wsum_b = reinterpret_cast<int*>(cand_b + W * kMaxSplatWords);     // [2][W]
    int* kcnt_b = wsum_b + 2 * W;                                          // [W][4]
    float* state_b = reinterpret_cast<float*>(reinterpret_cast<unsigned char*>(meta_off_b) + W * MS::kMetaBytes);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned* cand = cand_b + warp * kMaxSplatWords;
    __syncthreads();
    __shared__ float s_reach;
    const float reach2 = table_reach2(tab, ntot, &s_reach);
    unsigned int ev[7] = {0, 0, 0, 0, 0, 0, 0};
    unsigned int samples_c = 0;
    const int N = st.N;
    const long long npad = job.npad;
    // Block work units: the block's W warps take W consecutive chunks of 32 rays with the same segment,
    // frame and frequencies, and step through the samples together: within a sample, each group's
    // tests, its evaluations and the steps are separated by block barriers. Warps in the same phase share the
    // instruction cache lines of that phase (free-running warps in different phases thrashed it:
    // ncu "no instruction" stalls; 24% faster at 256x256, N = 1024, 3 frequencies, same results).
    __shared__ unsigned long long s_unit;
    __shared__ int s_kmax;
    const long long nbchunks = (job.nchunks + W - 1) / W;
    const long long btotal = nbchunks * job.nseg * job.nframes * job.nvc;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) { s_unit = atomicAdd(work, 1ull); s_kmax = 0; }
        __syncthreads();
        const unsigned long long u = s_unit;
        if (u >= (unsigned long long)btotal) break;
        const long long ur = btotal - 1 - (long long)u;             // last rays first
        const long long per_chunk = (long long)job.nseg * job.nframes * job.nvc;
        const long long w = (ur / per_chunk) * W + warp;
        const long long rem = ur % per_chunk;
        const int seg = int(rem / (job.nframes * job.nvc));
        const int y = int(rem % (job.nframes * job.nvc));
        const int f = y / job.nvc, v0 = (y % job.nvc) * CH;
        const long long j0 = w * 32 + lane;
        const bool live = j0 < job.npix;
        const long long j = live ? j0 : job.npix - 1;
        const int k0 = 1 + seg * job.seg_len;
        // the unit ends at the largest sample count of the block's rays (uneven counts)
        const int kmw = __reduce_max_sync(0xffffffffu, live ? int(P.get(PF_NSAMP, j)) : 0);
        if (lane == 0) atomicMax(&s_kmax, kmw);
        __syncthreads();
        const int kmax = s_kmax;
        const int k1 = min(min(N + 1, k0 + job.seg_len), kmax + 1);
        MixedSink<CH, KM, NT> sink;
        sink.tab = tab; sink.ntot = ntot; sink.knots = tab + ntot * ST_COUNT;
        sink.t_obs = float(ct[f]);
        sink.nc = min(CH, job.nfreq - v0);
        for (int c = 0; c < CH; ++c) {
            int v = min(v0 + c, job.nfreq - 1);
            double nh = cnu[v] / kNU0;
            sink.nu[c] = float(cnu[v]);
            sink.Lnu[c] = float(job.L / nh);
        }
        sink.a = float(st.a); sink.rh_lo = float(st.rh * (1 + 1e-3)); sink.dtau = float(P.get(PF_DTAU, j));
        sink.alpha = float(P.get(PF_ALPHA, j)); sink.beta = float(P.get(PF_BETA, j));
        sink.eta = float(P.get(PF_ETA, j)); sink.lam = float(P.get(PF_LAM, j));
        sink.a_sin_tho = float(st.a * sin(st.thetao)); sink.slab = job.slab; sink.nmax = job.nmax;
        sink.reach2 = reach2;
        sink.tid = threadIdx.x; sink.live = live;
        sink.nsamp = int(P.get(PF_NSAMP, j));
        sink.gstate = job.gstate; sink.gact = job.gact; sink.gnpad = npad; sink.jbase = (ur / per_chunk) * NT;
        sink.gN = N; sink.gframes = job.nframes; sink.gf = f; sink.gv0 = v0;
        sink.sf = sf_b;
        sink.items = reinterpret_cast<unsigned*>(items_b);
        sink.sres = reinterpret_cast<float*>(items_b);
        sink.res = res_b;
        sink.meta_off = meta_off_b;
        sink.meta_bits = meta_bits_b;
        sink.wsum = wsum_b;
        sink.scan_par = 0;
        sink.item_cap = W * MS::kItemBytes / 4;
        sink.sort_kinds = (KM != 1) || (job.nkv > 0);
        sink.kcnt = kcnt_b;
        sink.cand = cand;
        sink.state = state_b + threadIdx.x;
        sink.init();
        // the unit's samples in runs of cand_len, each with the candidate splats of its own box (a
        // segment's box spans the emission region in depth and keeps most of a large table)
        const int cl = job.cand_len > 0 ? job.cand_len : job.seg_len;
        const float* sp = stream + (long long)(k0 - 1) * SM_COUNT * npad + j;
        for (int kb = k0; kb < k1; kb += cl) {
            const int ke = min(k1, kb + cl);
            {
                UnitBox b = unit_box_empty();
                const float* bp = sp;
                for (int k = kb; k < ke; ++k, bp += SM_COUNT * npad) {
                    if (!live || k > sink.nsamp || !(__float_as_uint(bp[SM_FLAGS * npad]) & 8u)) continue;
                    const float x = bp[SM_X * npad], y = bp[SM_Y * npad], z = bp[SM_Z * npad];
                    if (x * x + y * y + z * z > reach2) continue;   // beyond every splat: no candidate needed
                    unit_box_add(b, x, y, z, sink.t_obs - bp[SM_T * npad]);
                }
                unit_box_reduce(b);
                unit_candidates(tab, ntot, b, lane, cand);
            }
            for (int k = kb; k < ke; ++k, sp += SM_COUNT * npad) {
                sink.kcur = k;
                const unsigned flags = __float_as_uint(sp[SM_FLAGS * npad]);
                sink.consume((flags & 8u) != 0u, sp[SM_X * npad], sp[SM_Y * npad], sp[SM_Z * npad], sp[SM_T * npad], sp[SM_R * npad],
                             sp[SM_STH * npad], sp[SM_CTH * npad], (flags & 2u) != 0u, (flags & 4u) != 0u);
            }
        }
        if (live) {
            for (int c = 0; c < sink.nc; ++c) {
                const float* S = sink.state + c * 20 * NT;
                float* o = seg_out + (((long long)((v0 + c) * job.nframes + f) * job.nseg + seg) * job.npix + j) * 20;
#pragma unroll
                for (int q = 0; q < 20; ++q) o[q] = S[q * NT];
            }
            for (int q = 0; q < 7; ++q) ev[q] += sink.ev[q];
            samples_c += sink.ev[0] * sink.nc;
        }
        __syncwarp();
    }
    if (counters) {
        atomicAdd(&counters[0], (unsigned long long)samples_c);
        for (int q = 1; q < 7; ++q) atomicAdd(&counters[q], (unsigned long long)ev[q]);
    }
}

// Front-to-back composition of a ray's segments and the observed Stokes vector (x nuhat^3).
__global__ void k_combine(MixedJob job, const double* __restrict__ cnu, const float* __restrict__ seg_out, double* __restrict__ out) {
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long ncombo = (long long)job.nframes * job.nfreq;
    if (q >= job.npix * ncombo) return;
    const long long combo = q / job.npix, j = q % job.npix;
    const float* base = seg_out + ((combo * job.nseg) * job.npix + j) * 20;
    double S[4];
    const float* last = base + (long long)(job.nseg - 1) * job.npix * 20;
    for (int r = 0; r < 4; ++r) S[r] = last[16 + r];
    for (int s = job.nseg - 2; s >= 0; --s) {
        const float* PS = base + (long long)s * job.npix * 20;
        double Sn[4];
        for (int r = 0; r < 4; ++r)
            Sn[r] = PS[16 + r] + PS[4 * r] * S[0] + PS[4 * r + 1] * S[1] + PS[4 * r + 2] * S[2] + PS[4 * r + 3] * S[3];
        for (int r = 0; r < 4; ++r) S[r] = Sn[r];
    }
    const int v = int(combo / job.nframes);
    const double nh = cnu[v] / kNU0, n3 = nh * nh * nh;
    double* o = out + (combo * job.npix + j) * 4;
    for (int r = 0; r < 4; ++r) o[r] = S[r] * n3;
}

}  // namespace ks
