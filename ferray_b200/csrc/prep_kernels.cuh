// prep_kernels.cuh -- operand preparation passes that feed the tensor-core
// kernels.  All are HBM-bound elementwise passes (one read, one or two
// writes per element) with grid-stride loops.
//
//  * split_bf16: x -> (hi, lo) with hi = bf16(x), lo = bf16(x - hi), both
//    round-to-nearest-even, for the 3xBF16 SGEMM (x = hi + lo + r,
//    |r| <= 2^-18 |x|); or three slices (hi, mid, lo), exact for f32, for the
//    6-product variant.  Optional complex real-embedding: the complex
//    product A*B equals the real product [Ar Ai] * [[Br Bi], [-Bi Br]],
//    whose columns are [Re C | Im C].
//  * split_i16: x -> (hi, lo) with x = 256*hi + lo, hi signed 8-bit,
//    lo unsigned 8-bit, for the byte-sliced i16 GEMM.
//  * pad_rows: copies a row-major byte matrix into a buffer whose row pitch
//    is a multiple of 16 bytes (TMA stride rule).
//  * row/column sums for the quantized GEMM's zero-point correction.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <cstdint>
#include <type_traits>

#include "fg_device.cuh"

namespace fg {

// Up to three bf16 slices: o[0] = bf16(x), o[s] = bf16(x - o[0] - ... - o[s-1]),
// every residual exact in f32.  Three slices hold all 24 bits of an f32.
struct BfPlanes {
    __nv_bfloat16* p[3];
};

__device__ __forceinline__ void split_n(float x, int ns, __nv_bfloat16 (&o)[3]) {
    float r = x;
#pragma unroll
    for (int s = 0; s < 3; ++s) {
        if (s < ns) {
            o[s] = __float2bfloat16_rn(r);
            r = r - __bfloat162float(o[s]);
        }
    }
}

__device__ __forceinline__ uint32_t pack_bf16x2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
    return static_cast<uint32_t>(__bfloat16_as_ushort(lo)) |
           (static_cast<uint32_t>(__bfloat16_as_ushort(hi)) << 16);
}

// ---- FP16 slices of power-of-two-scaled operands (split mode FP16).
// FP16 keeps 11 significant bits (BF16: 8), so two FP16 slices carry about
// 23 bits of an f32 against 17 for two BF16 slices, but FP16 spans only
// [2^-24, 65504].  Each operand is therefore multiplied by 2^s with s chosen
// from its largest magnitude so that max |x| 2^s lies in [2^14, 2^15): the hi
// slice cannot overflow, and an entry loses bits to the FP16 subnormal range
// only below 2^-38 of the operand's maximum.  The GEMM epilogue multiplies
// by 2^-(sA + sB).  Powers of two scale exactly (barring f32 under/overflow).

// hi = fp16(x), lo = fp16(x - hi), both round-to-nearest-even; the residual
// x - hi is exact in f32.
// A non-finite x keeps its Inf / NaN in hi with lo = 0.
__device__ __forceinline__ void split_f16x2(float x, uint16_t& hi, uint16_t& lo) {
    const __half h = __float2half_rn(x);
    hi = __half_as_ushort(h);
    const float hf = __half2float(h);
    lo = isfinite(hf) ? __half_as_ushort(__float2half_rn(x - hf)) : static_cast<uint16_t>(0);
}

// max |x| over the finite entries of a row-major stack of `count` rows x cols
// matrices (pitch ldx, matrices mstride apart), folded into *out with
// atomicMax on the float bits (non-negative floats order like their bit
// patterns).  Inf / NaN entries are left out, so they do not disable the
// scaling of the finite ones.  The caller zeroes *out.
__device__ __forceinline__ unsigned finite_abs_bits(float x) {
    return isfinite(x) ? __float_as_uint(fabsf(x)) : 0u;
}

static __global__ void amax_bits_kernel(const float* __restrict__ X, long long rows, long long cols,
                                        long long ldx, long long count, long long mstride,
                                        unsigned* __restrict__ out) {
    const bool vec = (cols % 4 == 0) && (ldx % 4 == 0) && (mstride % 4 == 0) &&
                     ((reinterpret_cast<uintptr_t>(X) & 15) == 0);
    const long long cq = vec ? cols / 4 : cols;
    const long long total = count * rows * cq;
    unsigned m = 0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long mr = e / cq, c = e - mr * cq;
        const long long z = mr / rows, r = mr - z * rows;
        const float* xr = X + z * mstride + r * ldx;
        if (vec) {
            const float4 w = __ldg(reinterpret_cast<const float4*>(xr) + c);
            m = max(m, max(max(finite_abs_bits(w.x), finite_abs_bits(w.y)),
                           max(finite_abs_bits(w.z), finite_abs_bits(w.w))));
        } else {
            m = max(m, finite_abs_bits(__ldg(xr + c)));
        }
    }
    m = __reduce_max_sync(0xFFFFFFFFu, m);
    __shared__ unsigned red[32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        unsigned v = threadIdx.x < (blockDim.x + 31) / 32 ? red[threadIdx.x] : 0u;
        v = __reduce_max_sync(0xFFFFFFFFu, v);
        if (threadIdx.x == 0 && v) atomicMax(out, v);
    }
}

// Real operand -> two FP16 planes of x 2^s (s from *amax), the layout of
// split_bf16_kernel_t: (row, 8-element group) pairs walked grid-stride, one
// 16-byte store per plane and group.
static __global__ void split_f16_kernel(const float* __restrict__ X, long long rows, long long cols,
                                        long long ldx, BfPlanes out, long long ldo, long long x_bstride,
                                        long long o_bstride, const unsigned* __restrict__ amax) {
    constexpr int U = 4;
    const int sc = f16_scale_exp(*amax);
    const float* Xb = X + blockIdx.y * x_bstride;
    const long long cq = (cols + 7) / 8;
    const long long total = rows * cq;
    const bool vec_in = (ldx % 4 == 0) && ((reinterpret_cast<uintptr_t>(Xb) & 15) == 0);
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e0 = blockIdx.x * (long long)blockDim.x + threadIdx.x; e0 < total; e0 += U * stride) {
        float v[U][8];
        long long rr[U], cc[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const long long e = e0 + u * stride;
            rr[u] = -1;
            cc[u] = 0;
            if (e < total) {
                const long long r = e / cq, c = (e - r * cq) * 8;
                rr[u] = r;
                cc[u] = c;
                const float* xr = Xb + r * ldx;
                if (vec_in && c + 7 < cols) {
                    const float4 w0 = __ldg(reinterpret_cast<const float4*>(xr + c));
                    const float4 w1 = __ldg(reinterpret_cast<const float4*>(xr + c + 4));
                    v[u][0] = w0.x; v[u][1] = w0.y; v[u][2] = w0.z; v[u][3] = w0.w;
                    v[u][4] = w1.x; v[u][5] = w1.y; v[u][6] = w1.z; v[u][7] = w1.w;
                } else {
#pragma unroll
                    for (int j = 0; j < 8; ++j) v[u][j] = (c + j < cols) ? xr[c + j] : 0.f;
                }
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (rr[u] < 0) break;
            uint32_t ph[4], pl[4];
#pragma unroll
            for (int j = 0; j < 8; j += 2) {
                uint16_t h0, l0, h1, l1;
                split_f16x2(mul_pow2(v[u][j], sc), h0, l0);
                split_f16x2(mul_pow2(v[u][j + 1], sc), h1, l1);
                ph[j / 2] = static_cast<uint32_t>(h0) | (static_cast<uint32_t>(h1) << 16);
                pl[j / 2] = static_cast<uint32_t>(l0) | (static_cast<uint32_t>(l1) << 16);
            }
            const long long off = blockIdx.y * o_bstride + rr[u] * ldo + cc[u];
            *reinterpret_cast<uint4*>(out.p[0] + off) = make_uint4(ph[0], ph[1], ph[2], ph[3]);
            *reinterpret_cast<uint4*>(out.p[1] + off) = make_uint4(pl[0], pl[1], pl[2], pl[3]);
        }
    }
}

// Complex operands for FP16 slices: the real embeddings of
// split_bf16_cplx_a_kernel / split_bf16_cplx_b_kernel, scaled by 2^s.
static __global__ void split_f16_cplx_a_kernel(const float2* __restrict__ A, long long M, long long K,
                                               long long lda, BfPlanes out, long long ldo,
                                               const unsigned* __restrict__ amax) {
    const int sc = f16_scale_exp(*amax);
    uint16_t* p0 = reinterpret_cast<uint16_t*>(out.p[0]);
    uint16_t* p1 = reinterpret_cast<uint16_t*>(out.p[1]);
    const long long total = M * K;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long r = e / K, c = e - r * K;
        const float2 v = A[r * lda + c];
        uint16_t hr, lr, hi, li;
        split_f16x2(mul_pow2(v.x, sc), hr, lr);
        split_f16x2(mul_pow2(v.y, sc), hi, li);
        p0[r * ldo + c] = hr;
        p1[r * ldo + c] = lr;
        p0[r * ldo + K + c] = hi;
        p1[r * ldo + K + c] = li;
    }
}

static __global__ void split_f16_cplx_b_kernel(const float2* __restrict__ B, long long K, long long N,
                                               long long ldb, BfPlanes out, long long ldo,
                                               const unsigned* __restrict__ amax) {
    const int sc = f16_scale_exp(*amax);
    const long long total = K * N;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long r = e / N, c = e - r * N;
        const float2 v = B[r * ldb + c];
        uint16_t hr[2], hi[2];
        split_f16x2(mul_pow2(v.x, sc), hr[0], hr[1]);
        split_f16x2(mul_pow2(v.y, sc), hi[0], hi[1]);
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            uint16_t* P = reinterpret_cast<uint16_t*>(out.p[s]);
            P[r * ldo + c] = hr[s];                                   // Br
            P[r * ldo + N + c] = hi[s];                               // Bi
            P[(K + r) * ldo + c] = static_cast<uint16_t>(hi[s] ^ 0x8000u);  // -Bi (sign flip, exact)
            P[(K + r) * ldo + N + c] = hr[s];                         // Br
        }
    }
}

// Real operand: X (rows x cols, pitch ldx) -> NS planes (pitch ldo, a
// multiple of 8).  The (row, 8-element group) pairs are flattened and
// walked grid-stride, four groups per thread per step (eight 16-byte loads in
// flight), each group written as one 16-byte store per plane.  NS is a
// template parameter and the slices are packed with integer ops, so nothing
// is indexed dynamically (no local memory).
template <int NS>
static __global__ void split_bf16_kernel_t(const float* __restrict__ X, long long rows, long long cols,
                                           long long ldx, BfPlanes out, long long ldo,
                                           long long x_bstride, long long o_bstride) {
    constexpr int U = 4;
    const float* Xb = X + blockIdx.y * x_bstride;
    const long long cq = (cols + 7) / 8;
    const long long total = rows * cq;
    const bool vec_in = (ldx % 4 == 0) && ((reinterpret_cast<uintptr_t>(Xb) & 15) == 0);
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e0 = blockIdx.x * (long long)blockDim.x + threadIdx.x; e0 < total; e0 += U * stride) {
        float v[U][8];
        long long rr[U], cc[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const long long e = e0 + u * stride;
            rr[u] = -1;
            cc[u] = 0;
            if (e < total) {
                const long long r = e / cq, c = (e - r * cq) * 8;
                rr[u] = r;
                cc[u] = c;
                const float* xr = Xb + r * ldx;
                if (vec_in && c + 7 < cols) {
                    const float4 w0 = __ldg(reinterpret_cast<const float4*>(xr + c));
                    const float4 w1 = __ldg(reinterpret_cast<const float4*>(xr + c + 4));
                    v[u][0] = w0.x; v[u][1] = w0.y; v[u][2] = w0.z; v[u][3] = w0.w;
                    v[u][4] = w1.x; v[u][5] = w1.y; v[u][6] = w1.z; v[u][7] = w1.w;
                } else {
#pragma unroll
                    for (int j = 0; j < 8; ++j) v[u][j] = (c + j < cols) ? xr[c + j] : 0.f;
                }
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (rr[u] < 0) break;
            uint32_t pk[NS][4];
#pragma unroll
            for (int j = 0; j < 8; j += 2) {
                __nv_bfloat16 a[3], b[3];
                split_n(v[u][j], NS, a);
                split_n(v[u][j + 1], NS, b);
#pragma unroll
                for (int s = 0; s < NS; ++s) pk[s][j / 2] = pack_bf16x2(a[s], b[s]);
            }
            const long long off = blockIdx.y * o_bstride + rr[u] * ldo + cc[u];
#pragma unroll
            for (int s = 0; s < NS; ++s)
                *reinterpret_cast<uint4*>(out.p[s] + off) = make_uint4(pk[s][0], pk[s][1], pk[s][2], pk[s][3]);
        }
    }
}

// Complex A (M x K, interleaved) -> real-embedded A' = [Ar | Ai] (M x 2K).
template <int NS>
static __global__ void split_bf16_cplx_a_kernel(const float2* __restrict__ A, long long M, long long K,
                                                long long lda, BfPlanes out, long long ldo) {
    const long long total = M * K;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        long long r = e / K, c = e - r * K;
        float2 v = A[r * lda + c];
        __nv_bfloat16 ore[3], oim[3];
        split_n(v.x, NS, ore);
        split_n(v.y, NS, oim);
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            out.p[s][r * ldo + c] = ore[s];
            out.p[s][r * ldo + K + c] = oim[s];
        }
    }
}

// Complex B (K x N) -> B' = [[Br, Bi], [-Bi, Br]] (2K x 2N).
template <int NS>
static __global__ void split_bf16_cplx_b_kernel(const float2* __restrict__ B, long long K, long long N,
                                                long long ldb, BfPlanes out, long long ldo) {
    const long long total = K * N;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        long long r = e / N, c = e - r * N;
        float2 v = B[r * ldb + c];
        __nv_bfloat16 ore[3], oim[3];
        split_n(v.x, NS, ore);
        split_n(v.y, NS, oim);
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            __nv_bfloat16* P = out.p[s];
            P[r * ldo + c] = ore[s];             // top-left      Br
            P[r * ldo + N + c] = oim[s];         // top-right     Bi
            P[(K + r) * ldo + c] = __hneg(oim[s]);  // bottom-left -Bi (exact)
            P[(K + r) * ldo + N + c] = ore[s];   // bottom-right  Br
        }
    }
}

static __global__ void split_i16_kernel(const int16_t* __restrict__ X, long long rows, long long cols,
                                 long long ldx, int8_t* __restrict__ hi, uint8_t* __restrict__ lo,
                                 long long ldo, long long x_bstride, long long o_bstride) {
    const int16_t* Xb = X + blockIdx.y * x_bstride;
    int8_t* hb = hi + blockIdx.y * o_bstride;
    uint8_t* lb = lo + blockIdx.y * o_bstride;
    const long long total = rows * cols;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        long long r = e / cols, c = e - r * cols;
        int v = Xb[r * ldx + c];
        hb[r * ldo + c] = static_cast<int8_t>(v >> 8);  // arithmetic shift: floor(v / 256)
        lb[r * ldo + c] = static_cast<uint8_t>(v & 0xFF);
    }
}

static __global__ void pad_rows_kernel(const uint8_t* __restrict__ X, long long rows, long long row_bytes,
                                long long ldx_bytes, uint8_t* __restrict__ Y, long long ldy_bytes,
                                long long x_bstride, long long y_bstride) {
    const uint8_t* Xb = X + blockIdx.y * x_bstride;
    uint8_t* Yb = Y + blockIdx.y * y_bstride;
    const long long total = rows * row_bytes;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        long long r = e / row_bytes, c = e - r * row_bytes;
        Yb[r * ldy_bytes + c] = Xb[r * ldx_bytes + c];
    }
}

// row_sum[i] = sum_k a[i, k] (u8), one warp per row, wrapping i32.  The
// warps stride over the rows, so a capped grid still writes every row.
static __global__ void row_sum_u8_kernel(const uint8_t* __restrict__ A, long long M, long long K,
                                  long long lda, int* __restrict__ out) {
    const int lane = threadIdx.x % 32;
    const long long warps = (long long)gridDim.x * blockDim.x / 32;
    for (long long row = (blockIdx.x * (long long)blockDim.x + threadIdx.x) / 32; row < M; row += warps) {
        uint32_t s = 0;
        for (long long k = lane; k < K; k += 32) s += A[row * lda + k];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
        if (lane == 0) out[row] = static_cast<int>(s);
    }
}

// col_sum[j] += sum over rows [y * rows_per, (y + 1) * rows_per) of b[k, j]
// (i8), y = blockIdx.y: one thread per column and row block, the partial
// sums added with atomicAdd into an array the caller zeroed.  Integer
// addition mod 2^32 is associative, so the result is exact and independent
// of the order the blocks arrive in.
static __global__ void col_sum_i8_kernel(const int8_t* __restrict__ B, long long K, long long N,
                                  long long ldb, long long rows_per, int* __restrict__ out) {
    const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= N) return;
    const long long k0 = blockIdx.y * rows_per, k1 = min(K, k0 + rows_per);
    uint32_t s = 0;
    for (long long k = k0; k < k1; ++k) s += static_cast<uint32_t>(static_cast<int32_t>(B[k * ldb + j]));
    atomicAdd(reinterpret_cast<unsigned int*>(out + j), s);
}

// C = beta * C for k == 0 (real / complex), and fill.
template <typename T>
static __global__ void scale_kernel(T* __restrict__ C, long long rows, long long cols, long long ldc,
                             T beta) {
    const long long total = rows * cols;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        long long r = e / cols, c = e - r * cols;
        C[r * ldc + c] = beta == T(0) ? T(0) : beta * C[r * ldc + c];
    }
}

// Split-K combine: ws holds `splits` partial products [s][z][M][N] (dense,
// s-major); C[z] = alpha * (ws[0] + ... + ws[S-1]) + beta * C[z] for floats
// (partials added in split order, round to nearest; beta == 0 leaves C
// unread), and C[z] = sum (+ C[z] when accumulate) mod 2^32 for int32.
template <typename T>
static __global__ void splitk_reduce_kernel(const T* __restrict__ ws, int splits, long long M,
                                            long long N, int batch, T* __restrict__ C,
                                            long long ldc, long long strideC, T alpha, T beta,
                                            int accumulate) {
    const long long mn = M * N, total = mn * batch, sstride = total;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long z = e / mn, rem = e - z * mn, r = rem / N, c = rem - r * N;
        T* dst = C + z * strideC + r * ldc + c;
        if constexpr (std::is_integral<T>::value) {  // int32
            uint32_t s = 0;
            for (int q = 0; q < splits; ++q) s += static_cast<uint32_t>(ws[q * sstride + e]);
            if (accumulate) s += static_cast<uint32_t>(*dst);
            *dst = static_cast<T>(s);
        } else {
            T s = ws[e];
            for (int q = 1; q < splits; ++q) s = s + ws[q * sstride + e];
            T o = alpha * s;
            if (beta != T(0)) o = fma(beta, *dst, o);
            *dst = o;
        }
    }
}

}  // namespace fg
