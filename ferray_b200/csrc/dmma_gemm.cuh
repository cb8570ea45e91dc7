// dmma_gemm.cuh -- plain DGEMM on the FP64 tensor path (mma.sync m8n8k4 f64,
// IEEE FP64 fused multiply-add per product, no reduced precision).
//
// tcgen05 has no FP64 kind, so FP64 matrix work on sm_100 runs either as
// DFMA (simt_gemm.cuh) or as DMMA warp-level MMAs.  One DMMA does 256 FP64
// FMAs per warp instruction, so the issue slots and registers that the DFMA
// kernel spends on 8 x 8 outer products are freed.
//
// CTA: 256 threads, 128 x 128 output tile, K blocks of 16, a 3-stage
// cp.async ring in shared memory (8-byte copies with zero fill past the
// matrix edges, so any leading dimension and alignment works).  Warps form
// a 2 (M) x 4 (N) grid of 64 x 32 warp tiles = 8 x 4 MMA tiles of 8 x 8.
// Fragments (m8n8k4, f64): A row = lane / 4, col = lane % 4; B row =
// lane % 4, col = lane / 4; C row = lane / 4, cols 2 (lane % 4) + {0, 1}.
// Shared layouts: A [m][k] with a 4-double pad (the 8 rows x 4 k of an A
// fragment fill 2 wavefronts exactly), B [k][n] with a 4-double pad.
// Batches and split-K follow simt_gemm_real: blockIdx.z = split * nbatch +
// batch index.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "simt_gemm.cuh"

namespace fg {

#ifndef FG_DMMA_BK
#define FG_DMMA_BK 16
#endif
// WARPS_M x WARPS_N warps, each MT x 4 MMA tiles of 8 x 8 (MT * 8 rows x 32
// columns); BM = WARPS_M * MT * 8, BN = WARPS_N * 32.
template <int WARPS_M_, int WARPS_N_, int MT_>
struct DmmaTile {
    static constexpr int WARPS_M = WARPS_M_, WARPS_N = WARPS_N_, MT = MT_;
    static constexpr int BM = WARPS_M * MT * 8, BN = WARPS_N * 32, BK = FG_DMMA_BK, STAGES = 3, THREADS = 256;
    static_assert(WARPS_M * WARPS_N == 8, "256 threads");
    static constexpr int APAD = 4, BPAD = 4;
    static constexpr int A_ELEMS = BM * (BK + APAD);
    static constexpr int B_ELEMS = BK * (BN + BPAD);
    static constexpr size_t SMEM = size_t(STAGES) * (A_ELEMS + B_ELEMS) * sizeof(double);
};
using DmmaCfg = DmmaTile<2, 4, 8>;        // 128 x 128, warps of 64 x 32
using DmmaSkinnyCfg = DmmaTile<1, 8, 4>;  // 32 x 256 for few rows, warps of 32 x 32

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool valid) {
    const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(s), "l"(gmem),
                 "r"(valid ? 8 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void dmma_8x8x4(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

template <class Cfg>
__global__ void __launch_bounds__(256, 1)
    dmma_gemm_f64_kernel(int M, int N, int K, double alpha, const double* __restrict__ A,
                         long long lda, const double* __restrict__ B, long long ldb, double beta,
                         double* __restrict__ C, long long ldc, BatchMap bm, int nbatch,
                         int ksplit) {
    constexpr int MT = Cfg::MT;
    extern __shared__ __align__(16) double dsm[];
    double* As = dsm;                                  // [STAGES][BM][BK + APAD]
    double* Bs = dsm + Cfg::STAGES * Cfg::A_ELEMS;     // [STAGES][BK][BN + BPAD]

    const int zb = blockIdx.z % nbatch, zs = blockIdx.z / nbatch;
    long long oa, ob;
    batch_offsets(bm, zb, oa, ob);
    const int k_begin = zs * ksplit;
    A += oa + k_begin;
    B += ob + (long long)k_begin * ldb;
    C += blockIdx.z * bm.c_bstride;
    K = min(K - k_begin, ksplit);

    const int tid = threadIdx.x, lane = tid % 32, warp = tid / 32;
    const int wm = warp / Cfg::WARPS_N, wn = warp % Cfg::WARPS_N;  // warps of MT * 8 x 32
    const int m0 = blockIdx.y * Cfg::BM, n0 = blockIdx.x * Cfg::BN;
    const int kblocks = (K + Cfg::BK - 1) / Cfg::BK;

    // global -> shared: BM*BK/256 A and BK*BN/256 B elements per thread per stage
    auto load_stage = [&](int stage, int kb) {
        const int k0 = kb * Cfg::BK;
        double* as = As + stage * Cfg::A_ELEMS;
        double* bs = Bs + stage * Cfg::B_ELEMS;
#pragma unroll
        for (int i = 0; i < Cfg::BM * Cfg::BK / 256; ++i) {
            const int e = tid + 256 * i;
            const int r = e / Cfg::BK, c = e % Cfg::BK;  // A: BK k per row
            const int gr = m0 + r, gk = k0 + c;
            const bool ok = gr < M && gk < K;
            cp_async8(as + r * (Cfg::BK + Cfg::APAD) + c, ok ? A + (long long)gr * lda + gk : A, ok);
        }
#pragma unroll
        for (int i = 0; i < Cfg::BK * Cfg::BN / 256; ++i) {
            const int e = tid + 256 * i;
            const int r = e / Cfg::BN, c = e % Cfg::BN;  // B: BN n per row
            const int gk = k0 + r, gn = n0 + c;
            const bool ok = gk < K && gn < N;
            cp_async8(bs + r * (Cfg::BN + Cfg::BPAD) + c, ok ? B + (long long)gk * ldb + gn : B, ok);
        }
    };

    double acc[MT][4][2];
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

#pragma unroll
    for (int s = 0; s < Cfg::STAGES - 1; ++s) {
        if (s < kblocks) load_stage(s, s);
        cp_async_commit();
    }
    const int fr = lane / 4, fc = lane % 4;
    for (int kb = 0; kb < kblocks; ++kb) {
        cp_async_wait<Cfg::STAGES - 2>();
        __syncthreads();  // stage kb landed for everyone; stage kb-1 is free
        {
            const int nk = kb + Cfg::STAGES - 1;
            if (nk < kblocks) load_stage(nk % Cfg::STAGES, nk);
            cp_async_commit();
        }
        const double* as = As + (kb % Cfg::STAGES) * Cfg::A_ELEMS;
        const double* bs = Bs + (kb % Cfg::STAGES) * Cfg::B_ELEMS;
#pragma unroll
        for (int kk = 0; kk < Cfg::BK; kk += 4) {
            double af[MT], bf[4];
#pragma unroll
            for (int i = 0; i < MT; ++i)
                af[i] = as[(wm * MT * 8 + i * 8 + fr) * (Cfg::BK + Cfg::APAD) + kk + fc];
#pragma unroll
            for (int j = 0; j < 4; ++j)
                bf[j] = bs[(kk + fc) * (Cfg::BN + Cfg::BPAD) + wn * 32 + j * 8 + fr];
#pragma unroll
            for (int i = 0; i < MT; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) dmma_8x8x4(acc[i][j], af[i], bf[j]);
        }
    }
    cp_async_wait<0>();

#pragma unroll
    for (int i = 0; i < MT; ++i) {
        const int r = m0 + wm * MT * 8 + i * 8 + fr;
        if (r >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int c = n0 + wn * 32 + j * 8 + 2 * fc;
            double* p = C + (long long)r * ldc + c;
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                if (c + u < N) {
                    double v = alpha * acc[i][j][u];
                    if (beta != 0.0) v = fma(beta, p[u], v);
                    p[u] = v;
                }
            }
        }
    }
}

// ZGEMM as a real GEMM: interleaved complex A (M x K) is the real matrix
// A' = [ar0 ai0 ar1 ai1 ...] (M x 2K) as it lies in memory; B' (2K x 2N) holds
// the 2 x 2 block [[br, bi], [-bi, br]] for every complex b, so row i of A'
// times columns 2n and 2n+1 of B' give Re and Im of (AB)[i, n], and C'
// (M x 2N) is C interleaved.  This pass writes B' (pitch 2N).
static __global__ void zgemm_expand_b_kernel(const double2* __restrict__ B, long long K, long long N,
                                             long long ldb, double* __restrict__ Bx) {
    const long long total = K * N;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long k = e / N, n = e - k * N;
        const double2 b = B[k * ldb + n];
        double* r0 = Bx + (2 * k) * (2 * N) + 2 * n;
        double* r1 = r0 + 2 * N;
        *reinterpret_cast<double2*>(r0) = make_double2(b.x, b.y);
        *reinterpret_cast<double2*>(r1) = make_double2(-b.y, b.x);
    }
}

}  // namespace fg
