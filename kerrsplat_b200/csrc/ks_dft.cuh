// ks_dft.cuh -- the image-to-visibility DFT, its adjoint, and the frame chi^2 + seed
// (src/Fit/device_visibilities.jl:53-111).
//
// V_k = tap_k scale sum_j I_j exp(+2 pi i (u_k l_j + v_k m_j)), l = -(i - (na + 1)/2) psize (east is
// -alpha), m = (j - (nb + 1)/2) psize, for the four Stokes images at once. The reference evaluates it
// directly, one work item per baseline with a sincos per (baseline, pixel) (vis_kernel!, seed_kernel!);
// the plain FP64 path here does the same. The mixed path uses the separable form
//     T[(s, j), (k, c|s)] = sum_i I_s[i, j] (cos | sin)(2 pi u_k l_i)          (a GEMM, K = na)
//     V_k,s = tap_k scale sum_j exp(2 pi i v_k m_j) (T_c + i T_s)[(s, j), k]    (a reduction over j)
// and the adjoint seed[i, (s, j)] = sum_k [cos . C_r + sin . C_i][i, k]         (a GEMM, K = 2 nuv)
// with C[k, (s, j)] = conj(exp(2 pi i v_k m_j)) w_k,s tap_k scale. The GEMMs run on the tensor cores in
// 3xTF32 (a = a_hi + a_lo, a_hi b_hi + a_hi b_lo + a_lo b_hi with FP32 accumulation; mma.sync m16n8k8).
// Twiddles are evaluated with the phase reduced in FP64 (sincospi of the fractional cycle).
#pragma once
#include <cuda_runtime.h>

namespace ksdft {

constexpr double kPi = 3.141592653589793238462643383279502884;

// out[x][2k + c] = (cos | sin)(2 pi f_k x), rows x = 0..nx-1 with offset(x) = sign * (x + 1 - (nx + 1)/2) * psize
__global__ void k_twiddle(int nx, double sign, double psize, long long nf, const double* __restrict__ f, float* __restrict__ out, long long ld) {
    long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= (long long)nx * nf) return;
    long long x = q / nf, k = q % nf;
    double off = sign * (double(x + 1) - double(nx + 1) / 2.0) * psize;
    double cyc = f[k] * off;                 // phase in cycles
    double fr = cyc - rint(cyc);
    double s, c;
    sincospi(2.0 * fr, &s, &c);
    out[x * ld + 2 * k] = float(c);
    out[x * ld + 2 * k + 1] = float(s);
}

// image (npix x 4 doubles, screen order p = i + j na, or sorted with perm) -> A[(s nb + j) na + i] FP32
__global__ void k_pack_image(const double* __restrict__ img, const long long* __restrict__ inv_perm, int na, int nb, float* __restrict__ A) {
    long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    long long npix = (long long)na * nb;
    if (q >= npix * 4) return;
    long long p = q % npix;   // screen index
    int s = int(q / npix);
    long long src = inv_perm ? inv_perm[p] : p;
    long long i = p % na, j = p / na;
    A[((long long)s * nb + j) * na + i] = float(img[src * 4 + s]);
}

__device__ __forceinline__ unsigned tf32(float x) {
    unsigned y;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ void mma_tf32(float* d, const unsigned* a, const unsigned* b) {
    asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

constexpr int BM = 128, BN = 128, BK = 16, NTHREADS = 256;

// C[M x N] = A[M x K] B[K x N], all row-major FP32, 3xTF32 on the tensor cores. 8 warps in a 2 x 4
// grid, each owning a 64 x 32 tile of C (4 x 4 m16n8 fragments). Edges are zero-filled in shared memory.
__global__ void __launch_bounds__(NTHREADS) k_gemm_3xtf32(int M, int N, int K, const float* __restrict__ A, long long lda,
                                                          const float* __restrict__ B, long long ldb, float* __restrict__ C, long long ldc) {
    __shared__ float As[BK][BM + 4];   // transposed: As[k][m]
    __shared__ float Bs[BK][BN + 4];
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
        // A tile: 128 rows x 16 k -> 2048 values, 8 per thread
#pragma unroll
        for (int q = 0; q < (BM * BK) / NTHREADS; ++q) {
            int e = tid + q * NTHREADS;
            int r = e / BK, kk = e % BK;
            long long gm = m0 + r, gk = k0 + kk;
            As[kk][r] = (gm < M && gk < K) ? A[gm * lda + gk] : 0.f;
        }
#pragma unroll
        for (int q = 0; q < (BK * BN) / NTHREADS; ++q) {
            int e = tid + q * NTHREADS;
            int kk = e / BN, c = e % BN;
            long long gk = k0 + kk, gn = n0 + c;
            Bs[kk][c] = (gk < K && gn < N) ? B[gk * ldb + gn] : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int ks = 0; ks < BK; ks += 8) {
            unsigned ah[4][4], al[4][4], bh[4][2], bl[4][2];
#pragma unroll
            for (int mi = 0; mi < 4; ++mi) {
                const int rm = wm * 64 + mi * 16;
                float v[4] = {As[ks + t][rm + g], As[ks + t][rm + g + 8], As[ks + t + 4][rm + g], As[ks + t + 4][rm + g + 8]};
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    ah[mi][q] = tf32(v[q]);
                    al[mi][q] = tf32(v[q] - __uint_as_float(ah[mi][q]));
                }
            }
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) {
                const int cn = wn * 32 + ni * 8;
                float v[2] = {Bs[ks + t][cn + g], Bs[ks + t + 4][cn + g]};
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    bh[ni][q] = tf32(v[q]);
                    bl[ni][q] = tf32(v[q] - __uint_as_float(bh[ni][q]));
                }
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

// V[k][s] = tap_k scale sum_j (Bc + i Bs)[j][k] (Tc + i Ts)[(s, j)][k]  (complex, written as re, im doubles)
__global__ void k_vis_combine(int nb, long long nuv, const float* __restrict__ Tm, long long ldt, const float* __restrict__ Bv, long long ldb,
                              const double* __restrict__ tap, double scale, double* __restrict__ V) {
    long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= nuv * 4) return;
    long long k = q % nuv;
    int s = int(q / nuv);
    double re = 0.0, im = 0.0;
    for (int j = 0; j < nb; ++j) {
        double bc = Bv[(long long)j * ldb + 2 * k], bs = Bv[(long long)j * ldb + 2 * k + 1];
        const float* tr = Tm + ((long long)s * nb + j) * ldt + 2 * k;
        double tc = tr[0], ts = tr[1];
        re += bc * tc - bs * ts;
        im += bc * ts + bs * tc;
    }
    double f = (tap ? tap[k] : 1.0) * scale;
    V[(k * 4 + s) * 2] = re * f;
    V[(k * 4 + s) * 2 + 1] = im * f;
}

// The adjoint right-hand side: Cm[(2k + c) ld + s nb + j] = (C_r | C_i)[k][(s, j)],
// C = conj(exp(2 pi i v_k m_j)) w_k,s tap_k scale.
__global__ void k_seed_rhs(int nb, long long nuv, const float* __restrict__ Bv, long long ldb, const double* __restrict__ w,
                           const double* __restrict__ tap, double scale, float* __restrict__ Cm, long long ldc) {
    long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= nuv * 4 * nb) return;
    int j = int(q % nb);
    long long r = q / nb;
    int s = int(r % 4);
    long long k = r / 4;
    double f = (tap ? tap[k] : 1.0) * scale;
    double wr = w[(k * 4 + s) * 2] * f, wi = w[(k * 4 + s) * 2 + 1] * f;
    double bc = Bv[(long long)j * ldb + 2 * k], bs = Bv[(long long)j * ldb + 2 * k + 1];
    Cm[(2 * k) * ldc + (long long)s * nb + j] = float(bc * wr + bs * wi);
    Cm[(2 * k + 1) * ldc + (long long)s * nb + j] = float(bc * wi - bs * wr);
}

// seed[(i, (s, j))] -> out (npix x 4, screen order or sorted through perm)
__global__ void k_unpack_seed(const float* __restrict__ S, long long lds, int na, int nb, const long long* __restrict__ inv_perm,
                              double* __restrict__ out) {
    long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    long long npix = (long long)na * nb;
    if (q >= npix * 4) return;
    long long p = q % npix;
    int s = int(q / npix);
    long long i = p % na, j = p / na;
    long long dst = inv_perm ? inv_perm[p] : p;
    out[dst * 4 + s] = double(S[i * lds + (long long)s * nb + j]);
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
