// ozaki_kernels.cuh -- operand slicing for the INT8 Ozaki DGEMM / ZGEMM.
//
// Method (Ozaki, Ogita, Oishi error-free splitting, in the INT8 form of
// Ootomo/Ozaki/Yokota and Uchino/Ozaki/Imamura): every row i of A is scaled
// by 2^-e_i, with e_i the frexp exponent of max_k |a_ik|, so |a_ik 2^-e_i| < 1;
// the scaled value t is written as S signed base-128 digits by exact
// scale-and-truncate steps, t = sum_{s=1..S} d_s 128^-s + r, |d_s| <= 127,
// |r| < 128^-S, each digit plane stored as an int8 slice.  Before that the
// inner dimension is balanced: AB = (A D)(D^-1 B) with D = diag(2^shift_k)
// chosen from A's column maxima and B's row maxima, so a term a_ik b_kj is
// represented relative to magnitudes near its own rather than to the largest
// entry of its row (which is what keeps exponent-spread inputs accurate).  Columns of B likewise with
// their own exponents f_j.  Then
//     C_ij = 2^(e_i+f_j) sum_{s,t} 2^(-7(s+t)) (A_s B_t)_ij
// and the products A_s B_t are exact int32 GEMMs on the integer tensor cores.
// Pairs with s + t > S + 1 are dropped (each is below K * 2^-7S of
// row-max * col-max).
//
// Layouts chosen so every group d = s + t is ONE plain int8 GEMM over a
// concatenated K: A slices side by side, A_all = [A_1 | A_2 | ... | A_S]
// (M x S*Kp), and B slices stacked in reverse, B_all = [B_S; ...; B_1]
// (S*Kp x N).  Group d is then A_all[:, 0:(d-1)Kp] times the last (d-1)Kp
// rows of B_all, i.e. sum_{s=1..d-1} A_s B_{d-s}.
//
// Complex operands use the real embedding [Ar Ai] and [[Br Bi], [-Bi Br]]
// (M x 2K and 2K x 2N) while slicing.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace fg {

// |x| as ordered bits (monotone for non-negative doubles, NaN above Inf).
__device__ __forceinline__ unsigned long long abs_bits(double x) {
    return static_cast<unsigned long long>(__double_as_longlong(x)) & 0x7FFFFFFFFFFFFFFFull;
}

// 2^e with frexp(max) = m * 2^e, m in [0.5, 1); zero rows get 1, non-finite
// rows get NaN so their outputs come out NaN.
__device__ __forceinline__ double scale_from_max_bits(unsigned long long bits) {
    const double mx = __longlong_as_double(static_cast<long long>(bits));
    if (mx == 0.0) return 1.0;
    if (!isfinite(mx)) return __longlong_as_double(0x7FF8000000000000ll);
    int e;
    frexp(mx, &e);
    return ldexp(1.0, e);
}

// Block-wide max of one value per thread (blockDim.x a multiple of 32, at
// most 1024); every thread gets the result.
__device__ __forceinline__ unsigned long long block_max_u64(unsigned long long v) {
    __shared__ unsigned long long red[32];
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
    __syncthreads();  // red[] may still be read from the previous call
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    v = threadIdx.x < blockDim.x / 32 ? red[threadIdx.x] : 0ull;
    if (threadIdx.x < 32)
        for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
    if (threadIdx.x == 0) red[0] = v;
    __syncthreads();
    return red[0];
}

// Row maxima of a real (cplx = 0) or complex (cplx = 1: Re and Im) matrix,
// one block per row (blocks stride over the rows), so a row's loads are
// spread over the block's warps.
// `shift` (may be null) holds the balancing exponent of each K index: the row
// maxima are those of A * diag(2^shift).
static __global__ void ozaki_row_scale_kernel(const double* __restrict__ A, long long M,
                                              long long K, long long lda, int cplx,
                                              const int* __restrict__ shift,
                                              double* __restrict__ scale) {
    const long long len = cplx ? 2 * K : K;
    for (long long row = blockIdx.x; row < M; row += gridDim.x) {
        const double* r = A + row * (cplx ? 2 * lda : lda);
        unsigned long long mx = 0;
        for (long long k = threadIdx.x; k < len; k += blockDim.x) {
            const int sh = shift ? shift[cplx ? (k >> 1) : k] : 0;
            mx = max(mx, abs_bits(ldexp(r[k], sh)));
        }
        mx = block_max_u64(mx);
        if (threadIdx.x == 0) scale[row] = scale_from_max_bits(mx);
    }
}

// Column maxima, pass 1: each thread scans `rows_per` rows of one (complex:
// embedded) column and folds the result into colmax_bits with atomicMax.
// Real B: N columns.  Complex B: the embedded B' has 2N columns, column c < N
// holds (Br, -Bi) and c >= N holds (Bi, Br) -> both have max(|Br|, |Bi|) of
// complex column c mod N, so N maxima suffice.
// The column maxima are those of diag(2^-shift) * B (shift may be null).
static __global__ void ozaki_col_max_kernel(const double* __restrict__ B, long long K, long long N,
                                            long long ldb, int cplx, long long rows_per,
                                            const int* __restrict__ shift,
                                            unsigned long long* __restrict__ colmax_bits) {
    const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= N) return;
    const long long k0 = blockIdx.y * rows_per, k1 = min(K, k0 + rows_per);
    unsigned long long mx = 0;
    for (long long k = k0; k < k1; ++k) {
        const int sh = shift ? -shift[k] : 0;
        if (cplx) {
            const double2 v = reinterpret_cast<const double2*>(B)[k * ldb + j];
            mx = max(mx, max(abs_bits(ldexp(v.x, sh)), abs_bits(ldexp(v.y, sh))));
        } else {
            mx = max(mx, abs_bits(ldexp(B[k * ldb + j], sh)));
        }
    }
    atomicMax(colmax_bits + j, mx);
}

// Balancing of the inner dimension: AB = (A D)(D^-1 B) for D = diag(2^shift_k).
// Pass 1: column maxima of A (over rows, atomicMax of ordered bits).
static __global__ void ozaki_a_colmax_kernel(const double* __restrict__ A, long long M, long long K,
                                             long long lda, int cplx, long long rows_per,
                                             unsigned long long* __restrict__ out) {
    const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (k >= K) return;
    const long long i0 = blockIdx.y * rows_per, i1 = min(M, i0 + rows_per);
    unsigned long long mx = 0;
    for (long long i = i0; i < i1; ++i) {
        if (cplx) {
            const double2 v = reinterpret_cast<const double2*>(A)[i * lda + k];
            mx = max(mx, max(abs_bits(v.x), abs_bits(v.y)));
        } else {
            mx = max(mx, abs_bits(A[i * lda + k]));
        }
    }
    atomicMax(out + k, mx);
}

// Pass 2: row maxima of B, one block per row (blocks stride over the rows).
static __global__ void ozaki_b_rowmax_kernel(const double* __restrict__ B, long long K, long long N,
                                             long long ldb, int cplx,
                                             unsigned long long* __restrict__ out) {
    const long long len = cplx ? 2 * N : N;
    for (long long row = blockIdx.x; row < K; row += gridDim.x) {
        const double* r = B + row * (cplx ? 2 * ldb : ldb);
        unsigned long long mx = 0;
        for (long long j = threadIdx.x; j < len; j += blockDim.x) mx = max(mx, abs_bits(r[j]));
        mx = block_max_u64(mx);
        if (threadIdx.x == 0) out[row] = mx;
    }
}

// Pass 3: shift_k = floor((eB_k - eA_k) / 2), so column k of A D and row k of
// D^-1 B peak at about the same magnitude.  Zero or non-finite maxima: 0.
static __global__ void ozaki_shift_kernel(const unsigned long long* __restrict__ a_colmax,
                                          const unsigned long long* __restrict__ b_rowmax,
                                          long long K, int* __restrict__ shift) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < K;
         k += (long long)gridDim.x * blockDim.x) {
        const double ma = __longlong_as_double(static_cast<long long>(a_colmax[k]));
        const double mb = __longlong_as_double(static_cast<long long>(b_rowmax[k]));
        int sh = 0;
        if (ma > 0.0 && mb > 0.0 && isfinite(ma) && isfinite(mb)) {
            int ea, eb;
            frexp(ma, &ea);
            frexp(mb, &eb);
            const int d = eb - ea;
            sh = d >= 0 ? d / 2 : -((-d + 1) / 2);
        }
        shift[k] = sh;
    }
}

static __global__ void ozaki_col_scale_kernel(const unsigned long long* __restrict__ colmax_bits,
                                              long long N, double* __restrict__ scale) {
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < N;
         j += (long long)gridDim.x * blockDim.x)
        scale[j] = scale_from_max_bits(colmax_bits[j]);
}

// Signed base-128 digits of t = x / scale, |t| < 1, by repeated exact
// scaling and truncation: t = sum_s d_s 128^-(s+1) + r, |r| < 128^-S, all
// digits carrying the sign of x (each step is exact in FP64).
template <int S>
__device__ __forceinline__ void ozaki_digits(double x, double inv_scale, int8_t (&d)[S]) {
    double t = x * inv_scale;  // power-of-two scaling: exact
    if (!isfinite(t)) t = 0.0;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        t *= 128.0;
        const double q = trunc(t);
        t -= q;
        d[s] = static_cast<int8_t>(static_cast<int>(q));
    }
}

// A slices: A_all[i, s*Kp + k] = digit s of A[i, k] (s = 0 most significant);
// complex A is embedded as [Ar | Ai] (width 2K).  Kp >= width, padding zero.
// Chunked: this launch writes embedded columns [k0, k0 + Kp) of the plane.
template <int S>
__global__ void ozaki_slice_a_kernel(const double* __restrict__ A, long long M, long long K,
                                     long long lda, int cplx, const int* __restrict__ shift,
                                     const double* __restrict__ scale,
                                     int8_t* __restrict__ out, long long Kp, long long k0) {
    const long long W = cplx ? 2 * K : K;
    const long long total = M * Kp;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long i = e / Kp, kl = e - i * Kp, k = k0 + kl;
        double x = 0.0;
        if (k < W) {
            if (cplx) {
                const long long kk = k < K ? k : k - K;
                x = ldexp(A[2 * (i * lda + kk) + (k < K ? 0 : 1)], shift[kk]);
            } else {
                x = ldexp(A[i * lda + k], shift[k]);
            }
        }
        int8_t d[S];
        ozaki_digits<S>(x, 1.0 / scale[i], d);
        int8_t* o = out + i * (S * Kp) + kl;
#pragma unroll
        for (int s = 0; s < S; ++s) o[s * Kp] = d[s];
    }
}

// B slices stacked in reverse: B_all[(S-1-s)*Kp + k, j] = digit s of B[k, j].
// Complex B is embedded as [[Br, Bi], [-Bi, Br]] (2K x 2N); Np >= width.
// Chunked: this launch writes embedded rows [k0, k0 + Kp) of the planes.
template <int S>
__global__ void ozaki_slice_b_kernel(const double* __restrict__ B, long long K, long long N,
                                     long long ldb, int cplx, const int* __restrict__ shift,
                                     const double* __restrict__ scale,
                                     int8_t* __restrict__ out, long long Kp, long long Np,
                                     long long k0) {
    const long long H = cplx ? 2 * K : K;   // embedded rows
    const long long W = cplx ? 2 * N : N;   // embedded columns
    const long long total = Kp * Np;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long kl = e / Np, j = e - kl * Np, k = k0 + kl;
        double x = 0.0;
        double sc = 1.0;
        if (k < H && j < W) {
            if (cplx) {
                const bool top = k < K, left = j < N;
                const long long kk = top ? k : k - K, jj = left ? j : j - N;
                const double2 v = reinterpret_cast<const double2*>(B)[kk * ldb + jj];
                // top-left Br, top-right Bi, bottom-left -Bi, bottom-right Br
                x = ldexp(top ? (left ? v.x : v.y) : (left ? -v.y : v.x), -shift[kk]);
                sc = scale[jj];
            } else {
                x = ldexp(B[k * ldb + j], -shift[k]);
                sc = scale[j];
            }
        }
        int8_t d[S];
        ozaki_digits<S>(x, 1.0 / sc, d);
#pragma unroll
        for (int s = 0; s < S; ++s) out[((S - 1 - s) * Kp + kl) * Np + j] = d[s];
    }
}

// ---------------------------------------------------------------- scheme II
// Ozaki scheme II (Ozaki, Uchino, Imamura: integer emulation of FP64 GEMM by
// the Chinese remainder theorem).  After the same balancing and row / column
// scaling as the slices above, every entry becomes one integer
//     a'_ik = rint(2^P a_ik 2^sh_k / 2^e_i),  |a'| <= 2^P,
// exactly representable as a double (below 2^53 it is an integer, above it
// t 2^P already is one), and likewise b'_kj with 2^-sh_k / 2^f_j.  For
// pairwise coprime moduli m_1..m_n <= 256 with product Mp > 2 K 2^(2P), the
// exact C' = A'B' is fixed by its residues C' mod m_l = (A' mod m_l)
// (B' mod m_l) mod m_l: ONE int8 GEMM per modulus on symmetric residues in
// [-128, 127] (exact int32 accumulation for K < 2^17), against the S(S+1)/2
// slice products of scheme I.  C' is rebuilt from the residue bytes in
// double arithmetic (oz2_reconstruct_kernel) and scaled back by 2^(e_i +
// f_j - 2P).
struct Oz2Consts {
    int n, P;
    int m[24];
    double inv_m[24];
    uint32_t magic[24];         // ceil(2^32 / m_l)
    uint32_t c20[24], c40[24];  // 2^20 mod m_l, 2^40 mod m_l
    double inv_M;               // 1 / Mp, for the CRT quotient
    double W[24][4];  // Mp / m_l in base-2^40 digits (W[l][0] least significant)
    double Mc[4];     // Mp in base-2^40 digits
    double M_d;       // Mp rounded to double
};

// Symmetric residue of the integer-valued double x (|x| <= 2^61) modulo m:
// q = rint(x / m) is off by at most one, r = x - q m is exact (fma), and at
// most two corrections bring r into [-(m/2), m - 1 - (m/2)].
__device__ __forceinline__ int8_t oz2_residue(double x, int m, double inv_m) {
    const double q = rint(x * inv_m);
    int r = static_cast<int>(fma(-q, static_cast<double>(m), x));
    const int lo = -(m / 2), hi = lo + m - 1;
    r += r < lo ? m : 0;
    r += r < lo ? m : 0;
    r -= r > hi ? m : 0;
    r -= r > hi ? m : 0;
    return static_cast<int8_t>(r);
}

// An integer-valued double |a| <= 2^60 as a sign and three 20-bit limbs
// (integer arithmetic from here on: one conversion per element, not one per
// modulus).
struct Oz2Limbs {
    uint32_t u0, u1, u2;
    bool neg;
};

__device__ __forceinline__ Oz2Limbs oz2_limbs(double a) {
    const long long v = static_cast<long long>(a);  // exact: a is an integer
    const unsigned long long u = static_cast<unsigned long long>(v < 0 ? -v : v);
    return Oz2Limbs{static_cast<uint32_t>(u & 0xFFFFFu), static_cast<uint32_t>((u >> 20) & 0xFFFFFu),
                    static_cast<uint32_t>(u >> 40), v < 0};
}

// Symmetric residue of the limbs' integer modulo m: x = u2 (2^40 mod m) +
// u1 (2^20 mod m) + u0 < 2^30, x mod m by a multiply-high with
// ceil(2^32 / m) (quotient exact or one too large) and one correction, then
// the sign and the symmetric range [-(m/2), m - 1 - (m/2)].
__device__ __forceinline__ uint32_t oz2_residue_limbs(const Oz2Limbs& a, uint32_t m, uint32_t magic,
                                                      uint32_t c20, uint32_t c40) {
    const uint32_t x = a.u2 * c40 + a.u1 * c20 + a.u0;
    int r = static_cast<int>(x - __umulhi(x, magic) * m);
    r += r < 0 ? static_cast<int>(m) : 0;  // r in [0, m)
    if (a.neg) r = r ? static_cast<int>(m) - r : 0;
    const int hi = static_cast<int>(m) - 1 - static_cast<int>(m / 2);
    r -= r > hi ? static_cast<int>(m) : 0;
    return static_cast<uint32_t>(r) & 0xFFu;
}

// Eight consecutive residues of one plane packed into 8 bytes.
__device__ __forceinline__ uint2 oz2_pack8(const Oz2Limbs (&x)[8], const Oz2Consts& c, int l) {
    const uint32_t m = static_cast<uint32_t>(c.m[l]), magic = c.magic[l], c20 = c.c20[l], c40 = c.c40[l];
    uint32_t w[2] = {0u, 0u};
#pragma unroll
    for (int u = 0; u < 8; ++u) w[u / 4] |= oz2_residue_limbs(x[u], m, magic, c20, c40) << (8 * (u % 4));
    return make_uint2(w[0], w[1]);
}

// A residue planes: A_all[i, l*Kp + k] = a'_ik mod m_l (complex A embedded
// as [Ar | Ai], width 2K; columns past the width are zero).  A thread takes
// eight consecutive k of one row and writes 8 bytes per plane.
__global__ void oz2_residue_a_kernel(const double* __restrict__ A, long long M, long long K,
                                     long long lda, int cplx, const int* __restrict__ shift,
                                     const double* __restrict__ scale, int8_t* __restrict__ out,
                                     long long Kp, const __grid_constant__ Oz2Consts c) {
    const long long W = cplx ? 2 * K : K;
    const long long K8 = Kp / 8, total = M * K8;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long i = e / K8, k0 = (e - i * K8) * 8;
        const double inv = 1.0 / scale[i];
        Oz2Limbs a[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const long long k = k0 + u;
            double x = 0.0;
            if (k < W) {
                if (cplx) {
                    const long long kk = k < K ? k : k - K;
                    x = ldexp(A[2 * (i * lda + kk) + (k < K ? 0 : 1)], shift[kk]);
                } else {
                    x = ldexp(A[i * lda + k], shift[k]);
                }
            }
            double v = rint(ldexp(x * inv, c.P));
            if (!isfinite(v)) v = 0.0;  // the row's NaN scale marks its outputs
            a[u] = oz2_limbs(v);
        }
        int8_t* o = out + i * (c.n * Kp) + k0;
        for (int l = 0; l < c.n; ++l) *reinterpret_cast<uint2*>(o + l * Kp) = oz2_pack8(a, c, l);
    }
}

// B residue planes: B_all[l*Kp + k, j] = b'_kj mod m_l (complex B embedded
// as [[Br, Bi], [-Bi, Br]]).  A thread takes eight consecutive j of one row.
__global__ void oz2_residue_b_kernel(const double* __restrict__ B, long long K, long long N,
                                     long long ldb, int cplx, const int* __restrict__ shift,
                                     const double* __restrict__ scale, int8_t* __restrict__ out,
                                     long long Kp, long long Np, const __grid_constant__ Oz2Consts c) {
    const long long H = cplx ? 2 * K : K, Wn = cplx ? 2 * N : N;
    const long long N8 = Np / 8, total = Kp * N8;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long k = e / N8, j0 = (e - k * N8) * 8;
        Oz2Limbs b[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const long long j = j0 + u;
            double x = 0.0, sc = 1.0;
            if (k < H && j < Wn) {
                if (cplx) {
                    const bool top = k < K, left = j < N;
                    const long long kk = top ? k : k - K, jj = left ? j : j - N;
                    const double2 v = reinterpret_cast<const double2*>(B)[kk * ldb + jj];
                    x = ldexp(top ? (left ? v.x : v.y) : (left ? -v.y : v.x), -shift[kk]);
                    sc = scale[jj];
                } else {
                    x = ldexp(B[k * ldb + j], -shift[k]);
                    sc = scale[j];
                }
            }
            double v = rint(ldexp(x * (1.0 / sc), c.P));
            if (!isfinite(v)) v = 0.0;
            b[u] = oz2_limbs(v);
        }
        for (int l = 0; l < c.n; ++l)
            *reinterpret_cast<uint2*>(out + (l * Kp + k) * Np + j0) = oz2_pack8(b, c, l);
    }
}

// C from the residue bytes R[l][i, j] = (C'_ij mod m_l) y_l mod m_l:
// S = sum_l R_l Mp/m_l is summed exactly in four base-2^40 digit sums
// (each below 2^53), q = rint(S / Mp) (S / Mp < n, and |C'| < Mp / 4 keeps
// it far from a tie), C' = S - q Mp digit by digit (exact), the digits are
// balanced into [-2^39, 2^39) with exact int64 carries and C' is evaluated
// from the top digit down (relative error about 2^-52).  Then
// C = alpha 2^(e_i + f_j - 2P) C' (+ beta C).  Complex: embedded column
// j < N is Re of column j, j >= N Im of column j - N (interleaved C).
__device__ __forceinline__ double oz2_rebuild(double s0, double s1, double s2, double s3,
                                              const Oz2Consts& c) {
    const double est = ((s3 * 0x1p120 + s2 * 0x1p80) + s1 * 0x1p40) + s0;
    const double q = rint(est * c.inv_M);
    long long d0 = static_cast<long long>(fma(-q, c.Mc[0], s0));
    long long d1 = static_cast<long long>(fma(-q, c.Mc[1], s1));
    long long d2 = static_cast<long long>(fma(-q, c.Mc[2], s2));
    long long d3 = static_cast<long long>(fma(-q, c.Mc[3], s3));
    const long long half = 1ll << 39;
    long long cy = (d0 + half) >> 40;
    d0 -= cy << 40;
    d1 += cy;
    cy = (d1 + half) >> 40;
    d1 -= cy << 40;
    d2 += cy;
    cy = (d2 + half) >> 40;
    d2 -= cy << 40;
    d3 += cy;
    double x = static_cast<double>(d3);
    x = fma(x, 0x1p40, static_cast<double>(d2));
    x = fma(x, 0x1p40, static_cast<double>(d1));
    return fma(x, 0x1p40, static_cast<double>(d0));
}

// One thread per output (measured faster than 4 or 8 outputs a thread:
// the digit sums are FP64-bound and fewer registers keep more warps
// resident).  A residue byte r becomes the double r by the exact
// 2^52 + r - 2^52 bit trick.
__global__ void oz2_reconstruct_kernel(const uint8_t* __restrict__ R, long long M, long long Nw,
                                       long long plane, const double* __restrict__ rsc,
                                       const double* __restrict__ csc, double* __restrict__ C,
                                       long long ldc, int cplx_half, double alpha, double beta,
                                       const __grid_constant__ Oz2Consts c) {
    const long long total = M * Nw;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long i = e / Nw, j = e - i * Nw;
        double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
        for (int l = 0; l < c.n; ++l) {
            const double r = __hiloint2double(0x43300000, R[l * plane + e]) - 0x1p52;
            s0 = fma(r, c.W[l][0], s0);
            s1 = fma(r, c.W[l][1], s1);
            s2 = fma(r, c.W[l][2], s2);
            s3 = fma(r, c.W[l][3], s3);
        }
        const double x = oz2_rebuild(s0, s1, s2, s3, c);
        const long long jc = cplx_half > 0 ? (j < cplx_half ? j : j - cplx_half) : j;
        const double o = (x * (ldexp(rsc[i], -2 * c.P) * alpha)) * csc[jc];
        double* dst = cplx_half > 0 ? C + 2 * (i * ldc + jc) + (j < cplx_half ? 0 : 1) : C + i * ldc + j;
        *dst = beta != 0.0 ? fma(beta, *dst, o) : o;
    }
}

}  // namespace fg
