// ks_dft.cuh -- the image-to-visibility DFT, its adjoint, and the frame chi^2 + seed
// (src/Fit/device_visibilities.jl:53-111).
//
// V_k = tap_k scale sum_j I_j exp(+2 pi i (u_k l_j + v_k m_j)), l = -(i - (na + 1)/2) psize (east is
// -alpha), m = (j - (nb + 1)/2) psize, for the four Stokes images at once. The reference evaluates it
// directly, one work item per baseline with a sincos per (baseline, pixel) (vis_kernel!, seed_kernel!);
// the plain FP64 path here does the same. The mixed path uses the separable form
//     T[(s, j), (k, c|s)] = sum_i I_s[i, j] (cos | sin)(2 pi u_k l_i)          (a GEMM, K = na)
//     V_k,s = tap_k scale sum_j exp(2 pi i v_k m_j) (T_c + i T_s)[(s, j), k]    (a reduction over j)
// and the adjoint seed[(s, j), i] = sum_k [C_r . cos + C_i . sin][(s, j), k]   (a GEMM, K = 2 nuv)
// with C[k, (s, j)] = conj(exp(2 pi i v_k m_j)) w_k,s tap_k scale.
//
// The GEMMs run on the tensor cores in 3xTF32. Every operand x is stored split, x_hi = tf32(x) and
// x_lo = tf32(x - x_hi) (round to nearest), by the kernel that produces it, and C = A_lo B_hi^T +
// A_hi B_lo^T + A_hi B_hi^T accumulates in FP32. Both operands are K-major: C[M][N] = A[M][K] B[N][K]^T,
// row strides a multiple of 4 floats. k_gemm_tc (tcgen05: TMA tiles with the 128-byte swizzle, UMMA
// 128 x 128 x 8 into a TMEM accumulator) is the default; k_gemm_3xtf32 (mma.sync m16n8k8) reads the same
// split operands and is the checked fallback. Twiddles are evaluated with the phase reduced in FP64
// (sincospi of the fractional cycle).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace ksdft {

constexpr double kPi = 3.141592653589793238462643383279502884;

// Row stride (floats) of a split operand: a multiple of 4 floats (16 bytes, the tensor-map stride rule).
inline long long pad4(long long n) { return (n + 3) & ~3LL; }

__device__ __forceinline__ unsigned tf32(float x) {
    unsigned y;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(y) : "f"(x));
    return y;
}

// x = hi + lo up to 2^-22 |x|, both exactly representable in TF32
__device__ __forceinline__ void split_store(float* __restrict__ hi, float* __restrict__ lo, long long at, float x) {
    const float h = __uint_as_float(tf32(x));
    hi[at] = h;
    lo[at] = __uint_as_float(tf32(x - h));
}

// (cos, sin)(2 pi f x) at row x, offset(x) = sign * (x + 1 - (nx + 1)/2) * psize
__device__ __forceinline__ void twiddle(long long x, int nx, double sign, double psize, double fk, float* c, float* s) {
    const double off = sign * (double(x + 1) - double(nx + 1) / 2.0) * psize;
    const double cyc = fk * off;   // phase in cycles
    const double fr = cyc - rint(cyc);
    double sd, cd;
    sincospi(2.0 * fr, &sd, &cd);
    *c = float(cd);
    *s = float(sd);
}

// out[x][2k + c] = (cos | sin)(2 pi f_k offset(x)), rows x = 0..nx-1
__global__ void k_twiddle(int nx, double sign, double psize, long long nf, const double* __restrict__ f, float* __restrict__ out, long long ld) {
    long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= (long long)nx * nf) return;
    long long x = q / nf, k = q % nf;
    twiddle(x, nx, sign, psize, f[k], &out[x * ld + 2 * k], &out[x * ld + 2 * k + 1]);
}

// The same table as a split GEMM operand, [x][2k + c] (transposed = 0) or [2k + c][x] (transposed = 1);
// consecutive threads write consecutive addresses in either layout.
__global__ void k_twiddle_split(int nx, double sign, double psize, long long nf, const double* __restrict__ f, int transposed,
                                float* __restrict__ hi, float* __restrict__ lo, long long ld) {
    long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= (long long)nx * nf) return;
    const long long x = transposed ? q % nx : q / nf, k = transposed ? q / nx : q % nf;
    float c, s;
    twiddle(x, nx, sign, psize, f[k], &c, &s);
    split_store(hi, lo, transposed ? (2 * k) * ld + x : x * ld + 2 * k, c);
    split_store(hi, lo, transposed ? (2 * k + 1) * ld + x : x * ld + 2 * k + 1, s);
}

// image (npix x 4 doubles, screen order p = i + j na, or sorted with perm) -> split A[(s nb + j) lda + i];
// one thread per pixel (its four Stokes values are one 32-byte read)
__global__ void k_pack_image(const double* __restrict__ img, const long long* __restrict__ inv_perm, int na, int nb,
                             float* __restrict__ hi, float* __restrict__ lo, long long lda) {
    const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;   // screen index
    if (p >= (long long)na * nb) return;
    const long long src = inv_perm ? inv_perm[p] : p;
    double v[4];
    if ((reinterpret_cast<uintptr_t>(img) & 31) == 0) {
        const double4 I = *reinterpret_cast<const double4*>(img + src * 4);
        v[0] = I.x, v[1] = I.y, v[2] = I.z, v[3] = I.w;
    } else {
        for (int s = 0; s < 4; ++s) v[s] = img[src * 4 + s];
    }
    const long long i = p % na, j = p / na;
#pragma unroll
    for (int s = 0; s < 4; ++s) split_store(hi, lo, ((long long)s * nb + j) * lda + i, float(v[s]));
}

// ---- the mma.sync fallback ------------------------------------------------------------------------

__device__ __forceinline__ void mma_tf32(float* d, const unsigned* a, const unsigned* b) {
    asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

constexpr int BM = 128, BN = 128, BK = 16, NTHREADS = 256;

// C[M x N] = A[M x K] B[N x K]^T from split operands, 3xTF32 with mma.sync. 8 warps in a 2 x 4 grid,
// each owning a 64 x 32 tile of C (4 x 4 m16n8 fragments). Edges are zero-filled in shared memory.
__global__ void __launch_bounds__(NTHREADS) k_gemm_3xtf32(int M, int N, int K, const float* __restrict__ Ah, const float* __restrict__ Al,
                                                          long long lda, const float* __restrict__ Bh, const float* __restrict__ Bl,
                                                          long long ldb, float* __restrict__ C, long long ldc) {
    __shared__ float Ash[BK][BM + 4], Asl[BK][BM + 4];   // transposed: As[k][m]
    __shared__ float Bsh[BK][BN + 4], Bsl[BK][BN + 4];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp >> 2, wn = warp & 3;   // 2 x 4 warps
    const long long m0 = (long long)blockIdx.y * BM, n0 = (long long)blockIdx.x * BN;
    const int g = lane >> 2, t = lane & 3;
    float acc[4][4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.f;
    for (int k0 = 0; k0 < K; k0 += BK) {
        // 128 rows x 16 k of each operand: 2048 values, 8 per thread
#pragma unroll
        for (int q = 0; q < (BM * BK) / NTHREADS; ++q) {
            const int e = tid + q * NTHREADS;
            const int r = e / BK, kk = e % BK;
            const long long gk = k0 + kk, gm = m0 + r, gn = n0 + r;
            const bool am = gm < M && gk < K, bn = gn < N && gk < K;
            Ash[kk][r] = am ? Ah[gm * lda + gk] : 0.f;
            Asl[kk][r] = am ? Al[gm * lda + gk] : 0.f;
            Bsh[kk][r] = bn ? Bh[gn * ldb + gk] : 0.f;
            Bsl[kk][r] = bn ? Bl[gn * ldb + gk] : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int ks = 0; ks < BK; ks += 8) {
            unsigned ah[4][4], al[4][4], bh[4][2], bl[4][2];
#pragma unroll
            for (int mi = 0; mi < 4; ++mi) {
                const int rm = wm * 64 + mi * 16;
                const int rr[4] = {rm + g, rm + g + 8, rm + g, rm + g + 8}, kq[4] = {ks + t, ks + t, ks + t + 4, ks + t + 4};
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    ah[mi][q] = __float_as_uint(Ash[kq[q]][rr[q]]);
                    al[mi][q] = __float_as_uint(Asl[kq[q]][rr[q]]);
                }
            }
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) {
                const int cn = wn * 32 + ni * 8;
                bh[ni][0] = __float_as_uint(Bsh[ks + t][cn + g]);
                bh[ni][1] = __float_as_uint(Bsh[ks + t + 4][cn + g]);
                bl[ni][0] = __float_as_uint(Bsl[ks + t][cn + g]);
                bl[ni][1] = __float_as_uint(Bsl[ks + t + 4][cn + g]);
            }
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni) {
                    mma_tf32(acc[mi][ni], al[mi], bh[ni]);   // small terms first
                    mma_tf32(acc[mi][ni], ah[mi], bl[ni]);
                    mma_tf32(acc[mi][ni], ah[mi], bh[ni]);
                }
        }
        __syncthreads();
    }
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) {
            const long long r0 = m0 + wm * 64 + mi * 16 + g, c0 = n0 + wn * 32 + ni * 8 + 2 * t;
            if (r0 < M && c0 < N) C[r0 * ldc + c0] = acc[mi][ni][0];
            if (r0 < M && c0 + 1 < N) C[r0 * ldc + c0 + 1] = acc[mi][ni][1];
            if (r0 + 8 < M && c0 < N) C[(r0 + 8) * ldc + c0] = acc[mi][ni][2];
            if (r0 + 8 < M && c0 + 1 < N) C[(r0 + 8) * ldc + c0 + 1] = acc[mi][ni][3];
        }
}

// ---- the tcgen05 kernel -----------------------------------------------------------------------------
//
// One CTA of 128 threads per 128 x 128 tile of C. Shared memory holds TC_STAGES stages of four operand
// tiles (A_hi, A_lo, B_hi, B_lo), each 128 rows x 32 floats (128 bytes: one 128-byte swizzle atom per
// 8 rows), filled by TMA from this GPU's memory (no multicast) with zero fill past the edges of the
// matrices. Thread 0 issues the copies, thread 32 issues the MMAs (three UMMA 128 x 128 x 8 per 8 k:
// lo.hi, hi.lo, hi.hi) and commits each stage back to the copier; the accumulator lives in 128 TMEM
// columns and all four warps read it back (tcgen05.ld 32x32b, warp w owns lanes 32w..32w+31 = rows).
// Every wait is bounded by `wait_limit` SM clock cycles: a wait that gives up sets bit 2 of `errflag`,
// the block skips the epilogue, waits (bounded) for the copies it issued, frees its TMEM and returns.
constexpr int TC_BM = 128, TC_BN = 128, TC_BK = 32, TC_STAGES = 3, TC_THREADS = 128;
constexpr int TC_TILE = TC_BM * TC_BK * 4;                      // bytes of one operand tile
constexpr int TC_STAGE = 4 * TC_TILE;
constexpr int TC_BARS = 2 * TC_STAGES + 1;                      // full[S], empty[S], done
constexpr int TC_SMEM = 1024 + TC_STAGES * TC_STAGE + 8 * TC_BARS + 16;
constexpr int TC_TMEM_COLS = 128;
// instruction descriptor of kind::tf32: F32 accumulator (bits 4-5 = 1), A and B TF32 (bits 7-9, 10-12
// = 2), both K-major (bits 15, 16 = 0), N >> 3 at bits 17-22, M >> 4 at bits 24-28
constexpr uint32_t TC_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | (uint32_t(TC_BN >> 3) << 17) | (uint32_t(TC_BM >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long long limit) {
    const long long t0 = clock64();
    while (true) {
        uint32_t ok;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(ok)
                     : "r"(bar), "r"(parity)
                     : "memory");
        if (ok) return true;
        if (clock64() - t0 > limit) return false;
    }
}

// Shared-memory matrix descriptor of a K-major tile with the 128-byte swizzle: start address >> 4
// (bits 0-13), leading offset 1 (unused by swizzled K-major layouts, bits 16-29), stride between 8-row
// groups 1024 B >> 4 (bits 32-45), descriptor version 1 (bits 46-47), layout SWIZZLE_128B = 2 (bits 61-63).
// The k-th 8-column slice of the atom starts 32 k bytes further (the swizzle is applied to the address).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
    return uint64_t((addr & 0x3FFFFu) >> 4) | (uint64_t(1) << 16) | (uint64_t(1024 >> 4) << 32) | (uint64_t(1) << 46) | (uint64_t(2) << 61);
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                 :
                 : "r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
                 : "memory");
}

__device__ __forceinline__ void umma_tf32(uint32_t tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\ttcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
                 :
                 : "r"(tmem), "l"(a), "l"(b), "r"(TC_IDESC), "r"(accumulate)
                 : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

#define KS_R8(b) "=r"(r[b]), "=r"(r[b + 1]), "=r"(r[b + 2]), "=r"(r[b + 3]), "=r"(r[b + 4]), "=r"(r[b + 5]), "=r"(r[b + 6]), "=r"(r[b + 7])
// 32 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t* r) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : KS_R8(0), KS_R8(8), KS_R8(16), KS_R8(24)
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
#undef KS_R8

__global__ void __launch_bounds__(TC_THREADS, 1)
    k_gemm_tc(int M, int N, int K, const __grid_constant__ CUtensorMap tAh, const __grid_constant__ CUtensorMap tAl,
              const __grid_constant__ CUtensorMap tBh, const __grid_constant__ CUtensorMap tBl, float* __restrict__ C, long long ldc,
              long long wait_limit, int skip_copies, unsigned* __restrict__ errflag) {
    extern __shared__ unsigned char tc_smem[];
    const uint32_t raw = smem_u32(tc_smem);
    const uint32_t base = (raw + 1023u) & ~1023u;   // the swizzle atoms need 1024-byte alignment
    const uint32_t bars = base + TC_STAGES * TC_STAGE;
    volatile uint32_t* slots = reinterpret_cast<volatile uint32_t*>(tc_smem + (bars + 8 * TC_BARS - raw));   // [0] TMEM base, [1] stop
    const int tid = threadIdx.x, warp = tid >> 5;
    const int m0 = blockIdx.y * TC_BM, n0 = blockIdx.x * TC_BN;
    const int nkb = (K + TC_BK - 1) / TC_BK;
    const uint32_t done = bars + 8u * (2 * TC_STAGES);

    if (tid == 0) {
        for (int q = 0; q < TC_BARS; ++q) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bars + 8u * q) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        slots[1] = 0;
    }
    __syncwarp();
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(bars + 8u * TC_BARS), "r"(TC_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = slots[0];

    bool gave_up = false;
    int issued = 0;   // thread 0: k-blocks whose copies are in flight or landed
    if (tid == 0) {
        for (int kb = 0; kb < nkb; ++kb) {
            const int s = kb % TC_STAGES;
            if (kb >= TC_STAGES && !mbar_wait(bars + 8u * (TC_STAGES + s), uint32_t((kb / TC_STAGES - 1) & 1), wait_limit)) {
                gave_up = true;
                break;
            }
            if (slots[1]) break;   // the MMA thread gave up
            const uint32_t full = bars + 8u * s, st = base + s * TC_STAGE;
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(full), "r"(TC_STAGE) : "memory");
            if (skip_copies) continue;   // error-path test hook: the stage never fills
            const int kx = kb * TC_BK;
            tma_load_2d(st, &tAh, kx, m0, full);
            tma_load_2d(st + TC_TILE, &tAl, kx, m0, full);
            tma_load_2d(st + 2 * TC_TILE, &tBh, kx, n0, full);
            tma_load_2d(st + 3 * TC_TILE, &tBl, kx, n0, full);
            issued = kb + 1;
        }
    } else if (tid == 32) {
        for (int kb = 0; kb < nkb; ++kb) {
            const int s = kb % TC_STAGES;
            if (!mbar_wait(bars + 8u * s, uint32_t((kb / TC_STAGES) & 1), wait_limit)) {
                gave_up = true;
                slots[1] = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t st = base + s * TC_STAGE;
#pragma unroll
            for (int k = 0; k < TC_BK / 8; ++k) {
                const uint64_t ah = sw128_desc(st + 32 * k), al = sw128_desc(st + TC_TILE + 32 * k);
                const uint64_t bh = sw128_desc(st + 2 * TC_TILE + 32 * k), bl = sw128_desc(st + 3 * TC_TILE + 32 * k);
                umma_tf32(tmem, al, bh, (kb | k) != 0);   // small terms first
                umma_tf32(tmem, ah, bl, 1);
                umma_tf32(tmem, ah, bh, 1);
            }
            umma_commit(bars + 8u * (TC_STAGES + s));   // the stage is free once these MMAs complete
        }
        umma_commit(done);   // every MMA this thread issued
    }
    if (!mbar_wait(done, 0, wait_limit)) gave_up = true;
    if (gave_up) atomicOr(errflag, 2u);
    const int bad = __syncthreads_or(gave_up ? 1 : 0);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    __syncwarp();
    if (!bad) {
        const int row = m0 + warp * 32 + (tid & 31);
        const bool vec = (ldc & 3) == 0 && (reinterpret_cast<uintptr_t>(C) & 15) == 0;
#pragma unroll 1
        for (int ch = 0; ch < TC_BN / 32 && n0 + ch * 32 < N; ++ch) {
            uint32_t r[32];
            tmem_ld32(tmem + (uint32_t(warp * 32) << 16) + uint32_t(ch * 32), r);
            const int col = n0 + ch * 32;
            if (row < M) {
                float* out = C + (long long)row * ldc + col;
                if (vec && col + 32 <= N) {
#pragma unroll
                    for (int q = 0; q < 8; ++q)
                        reinterpret_cast<float4*>(out)[q] =
                            make_float4(__uint_as_float(r[4 * q]), __uint_as_float(r[4 * q + 1]), __uint_as_float(r[4 * q + 2]), __uint_as_float(r[4 * q + 3]));
                } else {
#pragma unroll
                    for (int q = 0; q < 32; ++q)
                        if (col + q < N) out[q] = __uint_as_float(r[q]);
                }
            }
        }
    } else if (tid == 0) {
        // copies still in flight into this block's shared memory land before it exits
        for (int kb = issued > TC_STAGES ? issued - TC_STAGES : 0; kb < issued; ++kb)
            mbar_wait(bars + 8u * (kb % TC_STAGES), uint32_t((kb / TC_STAGES) & 1), wait_limit);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    __syncwarp();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS) : "memory");
}

// V[k][s] = tap_k scale sum_j (Bc + i Bs)[j][k] (Tc + i Ts)[(s, j)][k]  (complex, written as re, im doubles).
// A block of 32 baselines x 8 row groups for one Stokes parameter (grid.y): each thread sums the rows
// j = g, g + 8, ... of its baseline in FP64, and the 8 partial sums are added in a fixed order.
constexpr int VC_K = 32, VC_G = 8;
__global__ void __launch_bounds__(VC_K* VC_G) k_vis_combine(int nb, long long nuv, const float* __restrict__ Tm, long long ldt,
                                                             const float* __restrict__ Bv, long long ldb, const double* __restrict__ tap,
                                                             double scale, double* __restrict__ V) {
    __shared__ double red[2][VC_G][VC_K];
    const int kl = threadIdx.x % VC_K, g = threadIdx.x / VC_K, s = blockIdx.y;
    const long long k = (long long)blockIdx.x * VC_K + kl;
    double re = 0.0, im = 0.0;
    if (k < nuv) {
        for (int j = g; j < nb; j += VC_G) {
            const float2 b = *reinterpret_cast<const float2*>(Bv + (long long)j * ldb + 2 * k);
            const float2 t = *reinterpret_cast<const float2*>(Tm + ((long long)s * nb + j) * ldt + 2 * k);
            re += double(b.x) * t.x - double(b.y) * t.y;
            im += double(b.x) * t.y + double(b.y) * t.x;
        }
    }
    red[0][g][kl] = re;
    red[1][g][kl] = im;
    __syncthreads();
    if (g == 0 && k < nuv) {
        for (int q = 1; q < VC_G; ++q) { re += red[0][q][kl]; im += red[1][q][kl]; }
        const double f = (tap ? tap[k] : 1.0) * scale;
        V[(k * 4 + s) * 2] = re * f;
        V[(k * 4 + s) * 2 + 1] = im * f;
    }
}

// The adjoint right-hand side, split and K-major: CT[(s nb + j) ld + 2k + c] = (C_r | C_i)[k][(s, j)],
// C = conj(exp(2 pi i v_k m_j)) w_k,s tap_k scale.
__global__ void k_seed_rhs(int nb, long long nuv, const float* __restrict__ Bv, long long ldb, const double* __restrict__ w,
                           const double* __restrict__ tap, double scale, float* __restrict__ hi, float* __restrict__ lo, long long ldc) {
    long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= nuv * 4 * nb) return;
    const long long k = q % nuv, sj = q / nuv;
    const int s = int(sj / nb), j = int(sj % nb);
    double f = (tap ? tap[k] : 1.0) * scale;
    double wr = w[(k * 4 + s) * 2] * f, wi = w[(k * 4 + s) * 2 + 1] * f;
    double bc = Bv[(long long)j * ldb + 2 * k], bs = Bv[(long long)j * ldb + 2 * k + 1];
    split_store(hi, lo, sj * ldc + 2 * k, float(bc * wr + bs * wi));
    split_store(hi, lo, sj * ldc + 2 * k + 1, float(bc * wi - bs * wr));
}

// seed S[(s nb + j) lds + i] -> out (npix x 4, screen order or sorted through perm); one thread per pixel
__global__ void k_unpack_seed(const float* __restrict__ S, long long lds, int na, int nb, const long long* __restrict__ inv_perm,
                              double* __restrict__ out) {
    const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (p >= (long long)na * nb) return;
    const long long i = p % na, j = p / na;
    const long long dst = inv_perm ? inv_perm[p] : p;
    double4 o;
    o.x = S[j * lds + i];
    o.y = S[((long long)nb + j) * lds + i];
    o.z = S[(2LL * nb + j) * lds + i];
    o.w = S[(3LL * nb + j) * lds + i];
    if ((reinterpret_cast<uintptr_t>(out) & 31) == 0) {
        *reinterpret_cast<double4*>(out + dst * 4) = o;
    } else {
        out[dst * 4] = o.x, out[dst * 4 + 1] = o.y, out[dst * 4 + 2] = o.z, out[dst * 4 + 3] = o.w;
    }
}

// The plain FP64 port of vis_kernel! (one thread per baseline, a sincos per pixel).
__global__ void k_vis_direct(int na, int nb, const double* __restrict__ img, const long long* __restrict__ inv_perm, long long nuv,
                             const double* __restrict__ u, const double* __restrict__ v, const double* __restrict__ tap, double psize,
                             double scale, double* __restrict__ V) {
    long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (k >= nuv) return;
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const double uk = u[k], vk = v[k];
    for (long long p = 0; p < (long long)na * nb; ++p) {
        long long i = p % na, j = p / na;
        double l = -(double(i + 1) - double(na + 1) / 2.0) * psize, m = (double(j + 1) - double(nb + 1) / 2.0) * psize;
        double s, c;
        sincos(2.0 * kPi * (uk * l + vk * m), &s, &c);
        const double* I = img + (inv_perm ? inv_perm[p] : p) * 4;
        for (int q = 0; q < 4; ++q) { acc[2 * q] += I[q] * scale * c; acc[2 * q + 1] += I[q] * scale * s; }
    }
    double f = tap ? tap[k] : 1.0;
    for (int q = 0; q < 8; ++q) V[k * 8 + q] = acc[q] * f;
}

// The plain FP64 port of seed_kernel! (one thread per pixel).
__global__ void k_seed_direct(int na, int nb, const long long* __restrict__ inv_perm, long long nuv, const double* __restrict__ w,
                              const double* __restrict__ u, const double* __restrict__ v, const double* __restrict__ tap, double psize,
                              double scale, double* __restrict__ out) {
    long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (p >= (long long)na * nb) return;
    long long i = p % na, j = p / na;
    double l = -(double(i + 1) - double(na + 1) / 2.0) * psize, m = (double(j + 1) - double(nb + 1) / 2.0) * psize;
    double acc[4] = {0, 0, 0, 0};
    for (long long k = 0; k < nuv; ++k) {
        double s, c;
        sincos(2.0 * kPi * (u[k] * l + v[k] * m), &s, &c);
        double f = scale * (tap ? tap[k] : 1.0);
        for (int q = 0; q < 4; ++q) {
            double wr = w[(k * 4 + q) * 2] * f, wi = w[(k * 4 + q) * 2 + 1] * f;
            acc[q] += wr * c + wi * s;   // Re[w e^{-i phi}]
        }
    }
    long long dst = inv_perm ? inv_perm[p] : p;
    for (int q = 0; q < 4; ++q) out[dst * 4 + q] = acc[q];
}

// Residuals, chi^2 partial sums (one per block, summed on the host in block order) and the adjoint
// weights w = 2 conj(g) r / sigma, r = (g V - d) / sigma, per (baseline, Stokes) (device_visibilities.jl:105-107).
__global__ void k_chi2_weights(long long nuv, const double* __restrict__ V, const double* __restrict__ g, const double* __restrict__ d,
                               const double* __restrict__ sigma, double* __restrict__ w, double* __restrict__ partial) {
    __shared__ double red[256];
    long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    double c2 = 0.0;
    if (q < nuv * 4) {
        long long k = q / 4;
        double gr = g ? g[2 * k] : 1.0, gi = g ? g[2 * k + 1] : 0.0;
        double vr = V[2 * q], vi = V[2 * q + 1];
        double sg = sigma[q];
        double rr = (gr * vr - gi * vi - d[2 * q]) / sg, ri = (gr * vi + gi * vr - d[2 * q + 1]) / sg;
        c2 = rr * rr + ri * ri;
        w[2 * q] = 2.0 * (gr * rr + gi * ri) / sg;      // 2 conj(g) r / sigma
        w[2 * q + 1] = 2.0 * (gr * ri - gi * rr) / sg;
    }
    red[threadIdx.x] = c2;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

}  // namespace ksdft
