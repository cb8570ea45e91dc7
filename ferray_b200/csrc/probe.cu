// probe.cu -- fg_probe_peak: the dense throughput each compute pipe reaches on
// this GPU, measured, so that every kernel's roofline fraction can be stated
// against a measured peak rather than a spec sheet.
//
// Each probe keeps one pipe busy on data that never leaves the SM:
//   FG_PROBE_INT8   tcgen05.mma.cta_group::1.kind::i8, M = 128, N = 256,
//                   K = 32 per instruction, operands in shared memory
//                   (pseudo-random bytes), s32 accumulator in TMEM;
//   FG_PROBE_BF16   the same with kind::f16, bf16 operands, f32 accumulator;
//   FG_PROBE_FP64   mma.sync m8n8k4 f64 (DMMA) on registers, 8 independent
//                   accumulators per warp;
//   FG_PROBE_FFMA   fmaf on registers, 8 independent chains per thread.
// One persistent grid over every SM, timed with CUDA events around the
// launch (launch and set-up are a few microseconds of a run of several
// milliseconds).  Operand values are random, not zero: a tensor core's power,
// and so its clock under the power cap, depends on the bits it multiplies.
// Every wait is bounded (tc_peak_kernel's final mbarrier wait, 4 s).
#include <cuda_runtime.h>

#include "runtime.h"
#include "tc_gemm.cuh"

namespace {

using namespace fg;

constexpr int kProbeThreads = 128;

struct alignas(1024) PeakSmem {
    uint8_t a[128 * 128];  // 128 rows x 128 bytes of K, 128-byte swizzled
    uint8_t b[256 * 128];  // 256 rows x 128 bytes of K
    uint64_t done;
    uint32_t tmem;
};

template <int KIND>
__global__ void __launch_bounds__(kProbeThreads, 1)
    tc_peak_kernel(int iters, DevStatus* status, unsigned long long timeout_ns) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    PeakSmem& s = *reinterpret_cast<PeakSmem*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    const int warp = threadIdx.x / 32;
    // pseudo-random operands (xorshift per word); for bf16 the exponent
    // field is kept moderate so products stay finite
    uint32_t x = 0x9E3779B9u ^ (blockIdx.x * 7919u + threadIdx.x * 104729u);
    for (int i = threadIdx.x; i < (128 * 128 + 256 * 128) / 4; i += blockDim.x) {
        x ^= x << 13;
        x ^= x >> 17;
        x ^= x << 5;
        uint32_t w = x;
        if (KIND == KIND_BF16) w = (w & 0x807F807Fu) | 0x3F003F00u;  // |v| in [0.5, 1)
        if (i < 128 * 128 / 4)
            reinterpret_cast<uint32_t*>(s.a)[i] = w;
        else
            reinterpret_cast<uint32_t*>(s.b)[i - 128 * 128 / 4] = w;
    }
    if (threadIdx.x == 0) {
        mbar_init(&s.done, 1);
        fence_mbar_init();
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic writes -> tensor core reads
    if (warp == 0) {
        tmem_alloc(&s.tmem, 256);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0 && elect_one()) {
        const uint32_t idesc = umma_idesc(KIND == KIND_I8 ? 2u : 1u, 1u, 1u, 0u, 0u, 128, 256);
        const uint32_t a0 = smem_u32(s.a), b0 = smem_u32(s.b);
        for (int it = 0; it < iters; ++it) {
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
                const uint64_t ad = umma_desc_sw128(a0 + kk * 32, 16, 1024);
                const uint64_t bd = umma_desc_sw128(b0 + kk * 32, 16, 1024);
                const uint32_t acc = (it > 0 || kk > 0) ? 1u : 0u;
                if constexpr (KIND == KIND_I8)
                    tc_mma_i8(s.tmem, ad, bd, idesc, acc);
                else
                    tc_mma_f16(s.tmem, ad, bd, idesc, acc);
            }
        }
        tc_commit(&s.done);
        volatile int never = 0;
        mbar_wait(&s.done, 0, timeout_ns, status, 0x71, &never);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(s.tmem, 256);
    }
}

__global__ void __launch_bounds__(256) dmma_peak_kernel(int iters, double* sink) {
    double acc[8][2];
    double a = 1.0 + 1e-3 * (threadIdx.x & 7), b = 1.0 - 1e-3 * (threadIdx.x >> 5);
#pragma unroll
    for (int q = 0; q < 8; ++q) acc[q][0] = acc[q][1] = 0.0;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int q = 0; q < 8; ++q)
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                         : "+d"(acc[q][0]), "+d"(acc[q][1])
                         : "d"(a), "d"(b));
    }
    double t = 0.0;
#pragma unroll
    for (int q = 0; q < 8; ++q) t += acc[q][0] + acc[q][1];
    if (t == 1234.5) sink[blockIdx.x] = t;  // keeps the loop
}

__global__ void __launch_bounds__(256) ffma_peak_kernel(int iters, float* sink) {
    float acc[8];
    const float a = 1.0f + 1e-4f * (threadIdx.x & 7), b = 1e-4f * (threadIdx.x >> 5);
#pragma unroll
    for (int q = 0; q < 8; ++q) acc[q] = 1e-3f * q;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int q = 0; q < 8; ++q) acc[q] = fmaf(acc[q], a, b);
    }
    float t = 0.f;
#pragma unroll
    for (int q = 0; q < 8; ++q) t += acc[q];
    if (t == 1234.5f) sink[blockIdx.x] = t;
}

}  // namespace

using namespace fgrt;

extern "C" fg_status fg_probe_peak(fg_ctx* ctx, int which, double* per_second) {
    if (!ctx || !per_second) return set_error(FG_ERR_INVALID, "null argument");
    FG_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const int sms = ctx->sm_count;
    cudaEvent_t e0, e1;
    FG_CUDA(cudaEventCreate(&e0));
    FG_CUDA(cudaEventCreate(&e1));
    Scratch sink;
    fg_status rc = sink.alloc(static_cast<size_t>(sms) * 16 * sizeof(double), st);
    double ops = 0;
    auto run = [&](auto launch) -> fg_status {
        launch();  // warm-up (clocks, module load)
        FG_CUDA(cudaGetLastError());
        FG_CUDA(cudaEventRecord(e0, st));
        launch();
        FG_CUDA(cudaEventRecord(e1, st));
        FG_CUDA(cudaEventSynchronize(e1));
        FG_CUDA(cudaGetLastError());
        return FG_OK;
    };
    if (rc == FG_OK) {
        switch (which) {
            case FG_PROBE_INT8:
            case FG_PROBE_BF16: {
                const int iters = 20000;  // ~5 ms (INT8) / ~6 ms (BF16) at spec rates
                const size_t smem = sizeof(PeakSmem) + 1024;
                auto kern = which == FG_PROBE_INT8 ? tc_peak_kernel<KIND_I8> : tc_peak_kernel<KIND_BF16>;
                FG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
                rc = run([&] {
                    kern<<<sms, kProbeThreads, smem, st>>>(iters, ctx->d_status, 4000000000ull);
                    count_launch();
                });
                // per instruction: 128 x 256 x K (K = 32 i8 / 16 bf16) MACs, 2 ops each
                ops = 2.0 * 128 * 256 * (which == FG_PROBE_INT8 ? 32 : 16) * 4.0 * iters * sms;
                break;
            }
            case FG_PROBE_FP64: {
                const int iters = 20000, blocks = 2 * sms;  // ~5 ms at 40 TFLOP/s
                rc = run([&] {
                    dmma_peak_kernel<<<blocks, 256, 0, st>>>(iters, static_cast<double*>(sink.p));
                    count_launch();
                });
                ops = 512.0 * 8 * iters * (blocks * 256 / 32);  // 8x8x4 FMAs per warp mma
                break;
            }
            case FG_PROBE_FFMA: {
                const int iters = 80000, blocks = 8 * sms;  // ~5 ms at 75 TFLOP/s
                rc = run([&] {
                    ffma_peak_kernel<<<blocks, 256, 0, st>>>(iters, static_cast<float*>(sink.p));
                    count_launch();
                });
                ops = 2.0 * 8 * iters * (double)blocks * 256;
                break;
            }
            default:
                rc = set_error(FG_ERR_INVALID, "fg_probe_peak: unknown pipe");
        }
    }
    float ms = 0;
    if (rc == FG_OK) {
        cudaError_t e = cudaEventElapsedTime(&ms, e0, e1);
        if (e != cudaSuccess) rc = cuda_error(e, "cudaEventElapsedTime");
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    FG_TRY(rc);
    FG_TRY(fg_sync(ctx, nullptr));  // a probe wait that ran out is reported here
    *per_second = ms > 0 ? ops / (ms * 1e-3) : 0;
    return FG_OK;
}
