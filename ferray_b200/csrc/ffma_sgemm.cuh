// ffma_sgemm.cuh -- plain SGEMM on FFMA with a cp.async shared-memory ring.
//
// The register tile and summation order are those of simt_gemm_real<float,
// 8, 8, 8> (128 x 128 CTA tile, 8 x 8 outputs a thread in two 64-apart
// halves per direction, one FMA per product, k ascending), so results are
// bit-identical to it; what changes is how operands reach shared memory.
// A is first transposed into a packed K x Mp scratch (Mp = M rounded up to
// 4, zero padded), so both operand tiles are rows of 16-byte chunks that
// `cp.async.cg` copies global -> shared without passing through registers,
// in a 3-stage ring of BK = 32 (one __syncthreads per K block; 101 KB, two
// CTAs per SM).  The freed registers and the ring keep the FFMA pipe fed
// (B200, 8192^3: 52.9 TFLOP/s, against 52.0 for a 4-stage ring of BK = 16
// on the same box and 36.8 for the register-staged kernel).
// B is read in place when it is 16-byte aligned with ldb and N multiples of
// 4, otherwise from a packed copy (pitch Np = N rounded up to 4).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "simt_gemm.cuh"

namespace fg {

struct FfmaCfg {
    static constexpr int BM = 128, BN = 128, BK = 32, STAGES = 3, THREADS = 256, PAD = 4;
    static constexpr int AS = BK * (BM + PAD), BS = BK * (BN + PAD);  // floats per stage
    static constexpr size_t SMEM = size_t(STAGES) * (AS + BS) * sizeof(float);
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
    const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem), "r"(valid ? 16 : 0)
                 : "memory");
}

// At[z] (K x ldat, zero beyond M) = A[z]^T for the `count` distinct A
// matrices (row-major M x K, leading dimension lda, matrix stride ms).
// Grid: x over 32-row blocks of M (padded), y over 32-column blocks of K,
// z over the matrices; 32 x 8 threads.
static __global__ void transpose_pack_kernel(const float* __restrict__ A, int M, int K, long long lda, long long ms,
                                             float* __restrict__ At, long long ldat) {
    __shared__ float t[32][33];
    const int m0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
    const float* a = A + blockIdx.z * ms;
    float* at = At + blockIdx.z * (long long)K * ldat;
    for (int i = threadIdx.y; i < 32; i += 8) {
        const int m = m0 + i, k = k0 + threadIdx.x;
        t[i][threadIdx.x] = (m < M && k < K) ? a[(long long)m * lda + k] : 0.f;
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += 8) {
        const int k = k0 + i, m = m0 + threadIdx.x;
        if (k < K && m < ldat) at[(long long)k * ldat + m] = t[threadIdx.x][i];
    }
}

// Bp[z] (K x ldp, zero beyond N) = B[z] (K x N, leading dimension ldb,
// matrix stride ms).
static __global__ void pack_rows_kernel(const float* __restrict__ B, int K, int N, long long ldb, long long ms,
                                        float* __restrict__ Bp, long long ldp) {
    const float* b = B + blockIdx.y * ms;
    float* bp = Bp + blockIdx.y * (long long)K * ldp;
    const long long total = (long long)K * ldp;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long k = e / ldp, n = e - k * ldp;
        bp[e] = n < N ? b[k * ldb + n] : 0.f;
    }
}

// CGEMM as a real GEMM (the ZGEMM embedding of dmma_gemm.cuh in f32):
// interleaved complex A (M x K) is the real M x 2K matrix it lies as, and
// B' (2K x 2N, pitch 2N) holds [[br, bi], [-bi, br]] for every complex b,
// so columns 2n and 2n + 1 of A B' are Re and Im of (AB)[:, n].
static __global__ void cgemm_expand_b_kernel(const float2* __restrict__ B, long long K, long long N, long long ldb,
                                             float* __restrict__ Bx) {
    const long long total = K * N;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long k = e / N, n = e - k * N;
        const float2 b = B[k * ldb + n];
        float* r0 = Bx + (2 * k) * (2 * N) + 2 * n;
        float* r1 = r0 + 2 * N;
        *reinterpret_cast<float2*>(r0) = make_float2(b.x, b.y);
        *reinterpret_cast<float2*>(r1) = make_float2(-b.y, b.x);
    }
}

// C = alpha At^T B + beta C.  At: packed K x ldat per A matrix (batch
// offsets from bm.a_bstride in packed elements); B: K x ldb with columns
// valid below `bcols` (a multiple of 4; chunks at or past it read zero).
// blockIdx.z = split * nbatch + batch index, as simt_gemm_real.
static __global__ void __launch_bounds__(FfmaCfg::THREADS, 2)
    ffma_sgemm_kernel(int M, int N, int K, float alpha, const float* __restrict__ At, long long ldat,
                      const float* __restrict__ B, long long ldb, int bcols, float beta, float* __restrict__ C,
                      long long ldc, BatchMap bm, int nbatch, int ksplit) {
    using Cfg = FfmaCfg;
    constexpr int BM = Cfg::BM, BN = Cfg::BN, BK = Cfg::BK, PAD = Cfg::PAD, STAGES = Cfg::STAGES;
    extern __shared__ __align__(16) float ffma_sm[];
    float* As = ffma_sm;                        // [STAGES][BK][BM + PAD]
    float* Bs = ffma_sm + STAGES * Cfg::AS;     // [STAGES][BK][BN + PAD]

    const int zb = blockIdx.z % nbatch, zs = blockIdx.z / nbatch;
    long long oa, ob;
    batch_offsets(bm, zb, oa, ob);
    const int k_begin = zs * ksplit;
    At += oa + (long long)k_begin * ldat;
    B += ob + (long long)k_begin * ldb;
    C += blockIdx.z * bm.c_bstride;
    K = min(K - k_begin, ksplit);

    const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int kblocks = (K + BK - 1) / BK;
    constexpr int CH = BK * BM / 4 / Cfg::THREADS;  // 16-byte chunks a thread copies per operand and stage

    auto load = [&](int stage, int kb) {
        const int k0 = kb * BK;
        float* as = As + stage * Cfg::AS;
        float* bs = Bs + stage * Cfg::BS;
#pragma unroll
        for (int i = 0; i < CH; ++i) {
            const int c = tid + Cfg::THREADS * i;
            const int r = c / (BM / 4), col = (c % (BM / 4)) * 4;
            const int gk = k0 + r;
            const int gm = m0 + col, gn = n0 + col;
            const bool oka = gk < K && gm < ldat;
            const bool okb = gk < K && gn < bcols;
            cp_async16(as + r * (BM + PAD) + col, oka ? At + (long long)gk * ldat + gm : At, oka);
            cp_async16(bs + r * (BN + PAD) + col, okb ? B + (long long)gk * ldb + gn : B, okb);
        }
    };

    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;

#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
        if (s < kblocks) load(s, s);
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    for (int kb = 0; kb < kblocks; ++kb) {
        asm volatile("cp.async.wait_group %0;" ::"n"(STAGES - 2) : "memory");
        __syncthreads();  // stage kb landed for all threads; stage kb - 1 is free
        {
            const int nk = kb + STAGES - 1;
            if (nk < kblocks) load(nk % STAGES, nk);
            asm volatile("cp.async.commit_group;" ::: "memory");
        }
        const float* as = As + (kb % STAGES) * Cfg::AS;
        const float* bs = Bs + (kb % STAGES) * Cfg::BS;
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            float af[8], bf[8];
            const float4 a0 = *reinterpret_cast<const float4*>(as + kk * (BM + PAD) + ty * 4);
            const float4 a1 = *reinterpret_cast<const float4*>(as + kk * (BM + PAD) + 64 + ty * 4);
            const float4 b0 = *reinterpret_cast<const float4*>(bs + kk * (BN + PAD) + tx * 4);
            const float4 b1 = *reinterpret_cast<const float4*>(bs + kk * (BN + PAD) + 64 + tx * 4);
            af[0] = a0.x; af[1] = a0.y; af[2] = a0.z; af[3] = a0.w;
            af[4] = a1.x; af[5] = a1.y; af[6] = a1.z; af[7] = a1.w;
            bf[0] = b0.x; bf[1] = b0.y; bf[2] = b0.z; bf[3] = b0.w;
            bf[4] = b1.x; bf[5] = b1.y; bf[6] = b1.z; bf[7] = b1.w;
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(af[i], bf[j], acc[i][j]);
        }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");

#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int r = m0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + (i - 4));
        if (r >= M) continue;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int c = n0 + (j < 4 ? tx * 4 + j : 64 + tx * 4 + (j - 4));
            if (c >= N) continue;
            float* p = C + (long long)r * ldc + c;
            float v = alpha * acc[i][j];
            if (beta != 0.f) v = fmaf(beta, *p, v);
            *p = v;
        }
    }
}

// Skinny form for few rows (M <= 32 per tile): a 32 x 256 CTA tile, each
// thread 2 consecutive rows x 16 columns (four 4-column groups 64 apart),
// the same cp.async ring and the same per-output k order (one FMA per
// product, k ascending), so it too is bit-identical to the 128 x 128
// kernels at equal split-K.  With few rows the work per B element is small,
// so the host splits K to fill the GPU.
struct FfmaSkinnyCfg {
    static constexpr int BM = 32, BN = 256, BK = 32, STAGES = 3, THREADS = 256, PAD = 4;
    static constexpr int AS = BK * (BM + PAD), BS = BK * (BN + PAD);
    static constexpr size_t SMEM = size_t(STAGES) * (AS + BS) * sizeof(float);
};

static __global__ void __launch_bounds__(FfmaSkinnyCfg::THREADS, 2)
    ffma_sgemm_skinny_kernel(int M, int N, int K, float alpha, const float* __restrict__ At, long long ldat,
                             const float* __restrict__ B, long long ldb, int bcols, float beta,
                             float* __restrict__ C, long long ldc, BatchMap bm, int nbatch, int ksplit) {
    using Cfg = FfmaSkinnyCfg;
    constexpr int BM = Cfg::BM, BN = Cfg::BN, BK = Cfg::BK, PAD = Cfg::PAD, STAGES = Cfg::STAGES;
    extern __shared__ __align__(16) float ffma_sk_sm[];
    float* As = ffma_sk_sm;                     // [STAGES][BK][BM + PAD]
    float* Bs = ffma_sk_sm + STAGES * Cfg::AS;  // [STAGES][BK][BN + PAD]

    const int zb = blockIdx.z % nbatch, zs = blockIdx.z / nbatch;
    long long oa, ob;
    batch_offsets(bm, zb, oa, ob);
    const int k_begin = zs * ksplit;
    At += oa + (long long)k_begin * ldat;
    B += ob + (long long)k_begin * ldb;
    C += blockIdx.z * bm.c_bstride;
    K = min(K - k_begin, ksplit);

    const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int kblocks = (K + BK - 1) / BK;
    constexpr int A_CH = BK * BM / 4;                  // 256 chunks: every thread takes one
    static_assert(A_CH <= Cfg::THREADS, "one A chunk per thread at most");
    constexpr int B_CH = BK * BN / 4 / Cfg::THREADS;   // 4 chunks a thread

    auto load = [&](int stage, int kb) {
        const int k0 = kb * BK;
        float* as = As + stage * Cfg::AS;
        float* bs = Bs + stage * Cfg::BS;
        if (tid < A_CH) {
            const int r = tid / (BM / 4), col = (tid % (BM / 4)) * 4;
            const int gk = k0 + r, gm = m0 + col;
            const bool ok = gk < K && gm < ldat;
            cp_async16(as + r * (BM + PAD) + col, ok ? At + (long long)gk * ldat + gm : At, ok);
        }
#pragma unroll
        for (int i = 0; i < B_CH; ++i) {
            const int c = tid + Cfg::THREADS * i;
            const int r = c / (BN / 4), col = (c % (BN / 4)) * 4;
            const int gk = k0 + r, gn = n0 + col;
            const bool ok = gk < K && gn < bcols;
            cp_async16(bs + r * (BN + PAD) + col, ok ? B + (long long)gk * ldb + gn : B, ok);
        }
    };

    float acc[2][16];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 16; ++j) acc[i][j] = 0.f;

#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
        if (s < kblocks) load(s, s);
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    for (int kb = 0; kb < kblocks; ++kb) {
        asm volatile("cp.async.wait_group %0;" ::"n"(STAGES - 2) : "memory");
        __syncthreads();
        {
            const int nk = kb + STAGES - 1;
            if (nk < kblocks) load(nk % STAGES, nk);
            asm volatile("cp.async.commit_group;" ::: "memory");
        }
        const float* as = As + (kb % STAGES) * Cfg::AS;
        const float* bs = Bs + (kb % STAGES) * Cfg::BS;
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            const float2 a2 = *reinterpret_cast<const float2*>(as + kk * (BM + PAD) + ty * 2);
            const float af[2] = {a2.x, a2.y};
            float bf[16];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float4 b = *reinterpret_cast<const float4*>(bs + kk * (BN + PAD) + q * 64 + tx * 4);
                bf[q * 4] = b.x; bf[q * 4 + 1] = b.y; bf[q * 4 + 2] = b.z; bf[q * 4 + 3] = b.w;
            }
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 16; ++j) acc[i][j] = fmaf(af[i], bf[j], acc[i][j]);
        }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");

#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const int r = m0 + ty * 2 + i;
        if (r >= M) continue;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int c = n0 + (j / 4) * 64 + tx * 4 + (j % 4);
            if (c >= N) continue;
            float* p = C + (long long)r * ldc + c;
            float v = alpha * acc[i][j];
            if (beta != 0.f) v = fmaf(beta, *p, v);
            *p = v;
        }
    }
}

}  // namespace fg
