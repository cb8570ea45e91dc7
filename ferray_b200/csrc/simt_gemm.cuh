// simt_gemm.cuh -- the plain (non-tensor-core) GEMMs: FP64 on the FP64 pipe
// (DFMA), FP32 on FFMA, and their complex forms by the 4M scheme
// (re += ar*br - ai*bi, im += ar*bi + ai*br, four FMAs per complex MAC).
//
// Register-blocked shared-memory kernels: a CTA of 256 threads owns a
// BM x BN tile of C; each thread accumulates TM x TN outputs in registers,
// split into two 64-apart halves in each direction so its shared-memory
// fragment loads are 16-byte vectors free of bank conflicts.  Global tiles
// are prefetched into registers one K block ahead and double-buffered in
// shared memory, so one __syncthreads per K block suffices.
//
// Batches: blockIdx.z is the output matrix; a BatchMap turns it into the
// operand matrices (NumPy broadcasting, stride 0 on broadcast dims).
#pragma once
#include <cuComplex.h>
#include <cuda_runtime.h>
#include <cstdint>

namespace fg {

struct BatchMap {
    int bdims;
    int bshape[4];
    long long a_bstride[4];  // elements
    long long b_bstride[4];
    long long c_bstride;     // elements between consecutive output matrices
};

__device__ __forceinline__ void batch_offsets(const BatchMap& bm, int bz, long long& oa,
                                              long long& ob) {
    oa = 0;
    ob = 0;
    int rem = bz;
    // unrolled over the 4 possible dims: constant indices keep the
    // parameter struct out of local memory
#pragma unroll
    for (int d = 3; d >= 0; --d) {
        if (d < bm.bdims) {
            const int idx = rem % bm.bshape[d];
            rem /= bm.bshape[d];
            oa += idx * bm.a_bstride[d];
            ob += idx * bm.b_bstride[d];
        }
    }
}

// ----------------------------------------------------------------- real
// Tile BM = 16 * TMM rows x BN = 16 * TNN columns on a 16 x 16 thread grid,
// TMM x TNN outputs per thread: 128 x 128 (8 x 8), 64 x 64 (4 x 4), and the
// skinny 32 x 128 (2 x 8) / 128 x 32 (8 x 2) for small M / small N.  Split-K: blockIdx.z = split * nbatch + batch index; split s
// covers K columns [s * ksplit, (s + 1) * ksplit) and writes output matrix
// blockIdx.z (the host points C at a partial-sum workspace then).
// Two resident blocks per SM except for the f64 128 x 128 tile, which needs
// more than 128 registers a thread.
template <typename T, int BK, int TMM, int TNN>
__global__ void __launch_bounds__(256, (sizeof(T) == 8 && TMM == 8 && TNN == 8) ? 1 : 2)
    simt_gemm_real(int M, int N, int K, T alpha, const T* __restrict__ A, long long lda,
                   const T* __restrict__ B, long long ldb, T beta, T* __restrict__ C,
                   long long ldc, BatchMap bm, int nbatch, int ksplit) {
    constexpr int BM = 16 * TMM, BN = 16 * TNN, PAD = 4, H = TMM / 2;
    // Columns of a thread: QN groups of GN contiguous elements (16 bytes),
    // group q at q * 16 * GN + tx * GN, so each 16-byte fragment load of a
    // half-warp reads 256 contiguous bytes (no bank conflicts for f64).
    constexpr int GN = 16 / sizeof(T) < TNN ? 16 / sizeof(T) : TNN, QN = TNN / GN;
    constexpr int A_PER = BM * BK / 256;  // A elements each thread loads per K block
    constexpr int B_PER = BK * BN / 256;
    __shared__ __align__(16) T As[2][BK][BM + PAD];
    __shared__ __align__(16) T Bs[2][BK][BN + PAD];

    const int zb = blockIdx.z % nbatch, zs = blockIdx.z / nbatch;
    long long oa, ob;
    batch_offsets(bm, zb, oa, ob);
    const int k_begin = zs * ksplit;
    A += oa + k_begin;
    B += ob + (long long)k_begin * ldb;
    C += blockIdx.z * bm.c_bstride;
    K = min(K - k_begin, ksplit);

    const int tid = threadIdx.x;
    const int tx = tid % 16, ty = tid / 16;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;

    // A loader: each thread reads A_PER consecutive k of one row.
    constexpr int A_TPR = BK / A_PER;  // threads per row
    const int a_r = tid / A_TPR, a_c = (tid % A_TPR) * A_PER;
    // B loader: each thread reads B_PER consecutive n of one k row.
    constexpr int B_TPR = BN / B_PER;
    const int b_r = tid / B_TPR, b_c = (tid % B_TPR) * B_PER;

    T ra[A_PER], rb[B_PER];
    auto load_global = [&](int k0) {
        const int gr = m0 + a_r;
#pragma unroll
        for (int j = 0; j < A_PER; ++j) {
            const int gk = k0 + a_c + j;
            ra[j] = (gr < M && gk < K) ? A[(long long)gr * lda + gk] : T(0);
        }
        const int gk = k0 + b_r;
#pragma unroll
        for (int j = 0; j < B_PER; ++j) {
            const int gn = n0 + b_c + j;
            rb[j] = (gk < K && gn < N) ? B[(long long)gk * ldb + gn] : T(0);
        }
    };
    auto store_shared = [&](int buf) {
#pragma unroll
        for (int j = 0; j < A_PER; ++j) As[buf][a_c + j][a_r] = ra[j];
#pragma unroll
        for (int j = 0; j < B_PER; ++j) Bs[buf][b_r][b_c + j] = rb[j];
    };

    T acc[TMM][TNN];
#pragma unroll
    for (int i = 0; i < TMM; ++i)
#pragma unroll
        for (int j = 0; j < TNN; ++j) acc[i][j] = T(0);

    const int kblocks = (K + BK - 1) / BK;
    load_global(0);
    store_shared(0);
    __syncthreads();
    for (int kb = 0; kb < kblocks; ++kb) {
        const int cur = kb & 1;
        if (kb + 1 < kblocks) load_global((kb + 1) * BK);
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            T af[TMM], bf[TNN];
#pragma unroll
            for (int i = 0; i < H; ++i) {
                af[i] = As[cur][kk][ty * H + i];
                af[H + i] = As[cur][kk][BM / 2 + ty * H + i];
            }
#pragma unroll
            for (int q = 0; q < QN; ++q)
#pragma unroll
                for (int g = 0; g < GN; ++g) bf[q * GN + g] = Bs[cur][kk][q * 16 * GN + tx * GN + g];
#pragma unroll
            for (int i = 0; i < TMM; ++i)
#pragma unroll
                for (int j = 0; j < TNN; ++j) acc[i][j] = fma(af[i], bf[j], acc[i][j]);
        }
        if (kb + 1 < kblocks) store_shared(cur ^ 1);
        __syncthreads();
    }

#pragma unroll
    for (int i = 0; i < TMM; ++i) {
        const int r = m0 + (i < H ? ty * H + i : BM / 2 + ty * H + (i - H));
        if (r >= M) continue;
#pragma unroll
        for (int j = 0; j < TNN; ++j) {
            const int c = n0 + (j / GN) * 16 * GN + tx * GN + (j % GN);
            if (c >= N) continue;
            T* p = C + (long long)r * ldc + c;
            T v = alpha * acc[i][j];
            if (beta != T(0)) v = fma(beta, *p, v);
            *p = v;
        }
    }
}

// ----------------------------------------------------------------- GEMV
// Matrix-vector forms of the plain real GEMM (HBM-bound: the matrix is read
// once).  matvec: N == 1, y = C[:, 0] = alpha * A x + beta * y with x = B[:, 0]
// (stride ldb); one warp per row, lanes stride over K with 16-byte loads when
// the row and x are contiguous and aligned, partial sums combined by a fixed
// butterfly.  vecmat: M == 1, y = C[0, :] = alpha * x B + beta * y with
// x = A[0, :]; a block owns 32 x G columns (16-byte loads along N), its 8
// warps take interleaved K rows and are summed in shared memory in warp
// order; blockIdx.y splits K (partials to a workspace, combined by
// splitk_reduce_kernel) when the columns alone do not fill the GPU.
template <typename T>
__global__ void __launch_bounds__(256)
    gemv_rows_kernel(int M, int K, T alpha, const T* __restrict__ A, long long lda,
                     const T* __restrict__ x, long long incx, T beta, T* __restrict__ y,
                     long long incy) {
    constexpr int G = 16 / sizeof(T);
    const int lane = threadIdx.x % 32;
    const long long row = (blockIdx.x * (long long)blockDim.x + threadIdx.x) / 32;
    if (row >= M) return;
    const T* a = A + row * lda;
    const bool vec = incx == 1 && (reinterpret_cast<uintptr_t>(a) % 16 == 0) &&
                     (reinterpret_cast<uintptr_t>(x) % 16 == 0);
    T acc[G];
#pragma unroll
    for (int g = 0; g < G; ++g) acc[g] = T(0);
    int k0 = 0;
    if (vec) {
        const int kv = K / G * G;
        for (int k = lane * G; k < kv; k += 32 * G) {
            T av[G], xv[G];
            if constexpr (sizeof(T) == 8) {
                const double2 p = *reinterpret_cast<const double2*>(a + k);
                const double2 q = *reinterpret_cast<const double2*>(x + k);
                av[0] = p.x; av[1] = p.y; xv[0] = q.x; xv[1] = q.y;
            } else {
                const float4 p = *reinterpret_cast<const float4*>(a + k);
                const float4 q = *reinterpret_cast<const float4*>(x + k);
                av[0] = p.x; av[1] = p.y; av[2] = p.z; av[3] = p.w;
                xv[0] = q.x; xv[1] = q.y; xv[2] = q.z; xv[3] = q.w;
            }
#pragma unroll
            for (int g = 0; g < G; ++g) acc[g] = fma(av[g], xv[g], acc[g]);
        }
        k0 = kv;
    }
    for (int k = k0 + lane; k < K; k += 32) acc[0] = fma(a[k], x[k * incx], acc[0]);
    T sum = acc[0];
#pragma unroll
    for (int g = 1; g < G; ++g) sum += acc[g];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xFFFFFFFFu, sum, o);
    if (lane == 0) {
        T* dst = y + row * incy;
        T v = alpha * sum;
        if (beta != T(0)) v = fma(beta, *dst, v);
        *dst = v;
    }
}

template <typename T>
__global__ void __launch_bounds__(256)
    gemv_cols_kernel(int N, int K, int ksplit, T alpha, const T* __restrict__ x, long long incx,
                     const T* __restrict__ B, long long ldb, T beta, T* __restrict__ y,
                     long long split_stride) {
    constexpr int G = 16 / sizeof(T);
    __shared__ T part[8][32 * G];
    const int lane = threadIdx.x % 32, warp = threadIdx.x / 32;
    const int c0 = blockIdx.x * 32 * G + lane * G;
    const int kb = blockIdx.y * ksplit, ke = min(K, kb + ksplit);
    const bool vec = c0 + G <= N && (ldb % G == 0) && (reinterpret_cast<uintptr_t>(B) % 16 == 0);
    T acc[G];
#pragma unroll
    for (int g = 0; g < G; ++g) acc[g] = T(0);
    for (int k = kb + warp; k < ke; k += 8) {
        const T xv = x[k * incx];
        const T* br = B + (long long)k * ldb + c0;
        if (vec) {
            if constexpr (sizeof(T) == 8) {
                const double2 p = *reinterpret_cast<const double2*>(br);
                acc[0] = fma(xv, p.x, acc[0]);
                acc[1] = fma(xv, p.y, acc[1]);
            } else {
                const float4 p = *reinterpret_cast<const float4*>(br);
                acc[0] = fma(xv, p.x, acc[0]); acc[1] = fma(xv, p.y, acc[1]);
                acc[2] = fma(xv, p.z, acc[2]); acc[3] = fma(xv, p.w, acc[3]);
            }
        } else {
#pragma unroll
            for (int g = 0; g < G; ++g)
                if (c0 + g < N) acc[g] = fma(xv, br[g], acc[g]);
        }
    }
#pragma unroll
    for (int g = 0; g < G; ++g) part[warp][lane * G + g] = acc[g];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int g = 0; g < G; ++g) {
            const int c = c0 + g;
            T sum = part[0][lane * G + g];
#pragma unroll
            for (int w = 1; w < 8; ++w) sum += part[w][lane * G + g];
            if (c < N) {
                if (gridDim.y > 1) {
                    y[blockIdx.y * split_stride + c] = sum;  // partial (alpha/beta in the combine)
                } else {
                    T v = alpha * sum;
                    if (beta != T(0)) v = fma(beta, y[c], v);
                    y[c] = v;
                }
            }
        }
    }
}

// ----------------------------------------------------------------- complex
template <typename T>
struct Cplx {
    T re, im;
};

// 4M complex GEMM: 64 x 64 complex tile, each thread 4 x 4 complex outputs.
template <typename T, int BK>
__global__ void __launch_bounds__(256)
    simt_gemm_cplx(int M, int N, int K, T alpha_re, T alpha_im, const Cplx<T>* __restrict__ A,
                   long long lda, const Cplx<T>* __restrict__ B, long long ldb, T beta_re,
                   T beta_im, Cplx<T>* __restrict__ C, long long ldc, BatchMap bm) {
    constexpr int BM = 64, BN = 64, PAD = 2;
    constexpr int A_PER = BM * BK / 256;
    constexpr int B_PER = BK * BN / 256;
    __shared__ __align__(16) T Asr[2][BK][BM + PAD];
    __shared__ __align__(16) T Asi[2][BK][BM + PAD];
    __shared__ __align__(16) T Bsr[2][BK][BN + PAD];
    __shared__ __align__(16) T Bsi[2][BK][BN + PAD];

    long long oa, ob;
    batch_offsets(bm, blockIdx.z, oa, ob);
    A += oa;
    B += ob;
    C += blockIdx.z * bm.c_bstride;

    const int tid = threadIdx.x;
    const int tx = tid % 16, ty = tid / 16;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    constexpr int A_TPR = BK / A_PER;
    const int a_r = tid / A_TPR, a_c = (tid % A_TPR) * A_PER;
    constexpr int B_TPR = BN / B_PER;
    const int b_r = tid / B_TPR, b_c = (tid % B_TPR) * B_PER;

    Cplx<T> ra[A_PER], rb[B_PER];
    auto load_global = [&](int k0) {
        const int gr = m0 + a_r;
#pragma unroll
        for (int j = 0; j < A_PER; ++j) {
            const int gk = k0 + a_c + j;
            ra[j] = (gr < M && gk < K) ? A[(long long)gr * lda + gk] : Cplx<T>{T(0), T(0)};
        }
        const int gk = k0 + b_r;
#pragma unroll
        for (int j = 0; j < B_PER; ++j) {
            const int gn = n0 + b_c + j;
            rb[j] = (gk < K && gn < N) ? B[(long long)gk * ldb + gn] : Cplx<T>{T(0), T(0)};
        }
    };
    auto store_shared = [&](int buf) {
#pragma unroll
        for (int j = 0; j < A_PER; ++j) {
            Asr[buf][a_c + j][a_r] = ra[j].re;
            Asi[buf][a_c + j][a_r] = ra[j].im;
        }
#pragma unroll
        for (int j = 0; j < B_PER; ++j) {
            Bsr[buf][b_r][b_c + j] = rb[j].re;
            Bsi[buf][b_r][b_c + j] = rb[j].im;
        }
    };

    T cr[4][4], ci[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) cr[i][j] = ci[i][j] = T(0);

    const int kblocks = (K + BK - 1) / BK;
    load_global(0);
    store_shared(0);
    __syncthreads();
    for (int kb = 0; kb < kblocks; ++kb) {
        const int cur = kb & 1;
        if (kb + 1 < kblocks) load_global((kb + 1) * BK);
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            T ar[4], ai[4], br[4], bi[4];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                ar[i] = Asr[cur][kk][ty * 2 + i];
                ar[2 + i] = Asr[cur][kk][32 + ty * 2 + i];
                ai[i] = Asi[cur][kk][ty * 2 + i];
                ai[2 + i] = Asi[cur][kk][32 + ty * 2 + i];
                br[i] = Bsr[cur][kk][tx * 2 + i];
                br[2 + i] = Bsr[cur][kk][32 + tx * 2 + i];
                bi[i] = Bsi[cur][kk][tx * 2 + i];
                bi[2 + i] = Bsi[cur][kk][32 + tx * 2 + i];
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    cr[i][j] = fma(ar[i], br[j], cr[i][j]);
                    cr[i][j] = fma(-ai[i], bi[j], cr[i][j]);
                    ci[i][j] = fma(ar[i], bi[j], ci[i][j]);
                    ci[i][j] = fma(ai[i], br[j], ci[i][j]);
                }
        }
        if (kb + 1 < kblocks) store_shared(cur ^ 1);
        __syncthreads();
    }

#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int r = m0 + (i < 2 ? ty * 2 + i : 32 + ty * 2 + (i - 2));
        if (r >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int c = n0 + (j < 2 ? tx * 2 + j : 32 + tx * 2 + (j - 2));
            if (c >= N) continue;
            Cplx<T>* p = C + (long long)r * ldc + c;
            T vr = alpha_re * cr[i][j] - alpha_im * ci[i][j];
            T vi = alpha_re * ci[i][j] + alpha_im * cr[i][j];
            if (beta_re != T(0) || beta_im != T(0)) {
                Cplx<T> o = *p;
                vr += beta_re * o.re - beta_im * o.im;
                vi += beta_re * o.im + beta_im * o.re;
            }
            *p = Cplx<T>{vr, vi};
        }
    }
}

}  // namespace fg
