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
// Tile BM = BN = 16 * TM (TM = 8: 128 x 128, TM = 4: 64 x 64 for small
// problems).  Split-K: blockIdx.z = split * nbatch + batch index; split s
// covers K columns [s * ksplit, (s + 1) * ksplit) and writes output matrix
// blockIdx.z (the host points C at a partial-sum workspace then).
// Two resident blocks per SM for the f32 128 x 128 tile (at most 128
// registers a thread); the f64 one needs more registers than that.
template <typename T, int BK, int TM>
__global__ void __launch_bounds__(256, (sizeof(T) == 4 && TM == 8) ? 2 : 1)
    simt_gemm_real(int M, int N, int K, T alpha, const T* __restrict__ A, long long lda,
                   const T* __restrict__ B, long long ldb, T beta, T* __restrict__ C,
                   long long ldc, BatchMap bm, int nbatch, int ksplit) {
    constexpr int BM = 16 * TM, BN = 16 * TM, PAD = 4, H = TM / 2;
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

    T acc[TM][TM];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TM; ++j) acc[i][j] = T(0);

    const int kblocks = (K + BK - 1) / BK;
    load_global(0);
    store_shared(0);
    __syncthreads();
    for (int kb = 0; kb < kblocks; ++kb) {
        const int cur = kb & 1;
        if (kb + 1 < kblocks) load_global((kb + 1) * BK);
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            T af[TM], bf[TM];
#pragma unroll
            for (int i = 0; i < H; ++i) {
                af[i] = As[cur][kk][ty * H + i];
                af[H + i] = As[cur][kk][BM / 2 + ty * H + i];
                bf[i] = Bs[cur][kk][tx * H + i];
                bf[H + i] = Bs[cur][kk][BN / 2 + tx * H + i];
            }
#pragma unroll
            for (int i = 0; i < TM; ++i)
#pragma unroll
                for (int j = 0; j < TM; ++j) acc[i][j] = fma(af[i], bf[j], acc[i][j]);
        }
        if (kb + 1 < kblocks) store_shared(cur ^ 1);
        __syncthreads();
    }

#pragma unroll
    for (int i = 0; i < TM; ++i) {
        const int r = m0 + (i < H ? ty * H + i : BM / 2 + ty * H + (i - H));
        if (r >= M) continue;
#pragma unroll
        for (int j = 0; j < TM; ++j) {
            const int c = n0 + (j < H ? tx * H + j : BN / 2 + tx * H + (j - H));
            if (c >= N) continue;
            T* p = C + (long long)r * ldc + c;
            T v = alpha * acc[i][j];
            if (beta != T(0)) v = fma(beta, *p, v);
            *p = v;
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
