// qmm_noalloc.cu -- fg_quantized_matmul_noalloc: the quantized u8 x i8 -> f32
// GEMM without any device allocation.
//
// Who needs it: callers that are not allowed to allocate device memory at
// call time -- a host whose device memory is owned by another allocator (a
// framework's caching pool that must account for every byte), a serving
// loop that admits work against a fixed HBM budget set at start-up, or a
// latency-critical loop that cannot afford the synchronisation and
// unbounded latency an allocation may bring.  fg_quantized_matmul needs
// (m + n) int32 of scratch for the zero-point row and column sums, which it
// takes from the stream-ordered allocator; this variant keeps that scratch
// in one fixed, file-scope device array instead.
//
// The array is kQmmNoAllocMaxM + kQmmNoAllocMaxN int32 (512 KiB) and lives
// in every GPU that loads this library until the process exits.  The first
// call on a device (with that device current) looks up the array's device
// address with cudaGetSymbolAddress; make that first call before any stream
// capture.  All calls share the array: the sum kernels overwrite every entry
// a call reads, so nothing has to start at zero, but calls whose kernels
// overlap on the GPU (different streams, or different host threads) race on
// it and must be serialised by the caller.
//
// Limits (anything else is rejected with FG_ERR_UNSUPPORTED and a message):
// m <= 65536, n <= 65536, k <= 65536 (exact int32 accumulation), and the
// operands must already meet the TMA rules -- 16-byte aligned a and b, k and
// n multiples of 16 -- because padding them would need scratch.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "prep_kernels.cuh"
#include "runtime.h"
#include "tc_gemm.cuh"

namespace {

constexpr long long kQmmNoAllocMaxM = 65536;
constexpr long long kQmmNoAllocMaxN = 65536;
constexpr long long kQmmNoAllocMaxK = 65536;
constexpr int kMaxDevices = 64;

// Row sums occupy [0, m), column sums [kQmmNoAllocMaxM, kQmmNoAllocMaxM + n).
static __device__ __align__(256) int g_qmm_sums[kQmmNoAllocMaxM + kQmmNoAllocMaxN];

using CfgQmmNoAlloc = fg::TcCfg<fg::KIND_I8, 256, 4, 1, 1, 1, 1, fg::EPI_QMM>;

std::mutex g_setup_mu;
int* g_sums_dev[kMaxDevices] = {nullptr};

// Once per device, with that device current: the device address of the
// scratch array (its name in host code is only a host-side stand-in) and
// the kernel's shared-memory opt-in.
fg_status setup_device(int device, int** out) {
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (g_sums_dev[device] == nullptr) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_qmm_sums);
        if (e != cudaSuccess) return fgrt::cuda_error(e, "cudaGetSymbolAddress(qmm scratch)");
        e = cudaFuncSetAttribute(fg::tc_gemm_kernel<CfgQmmNoAlloc>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(fg::tc_smem_bytes<CfgQmmNoAlloc>()));
        if (e != cudaSuccess) return fgrt::cuda_error(e, "cudaFuncSetAttribute(qmm no-alloc)");
        g_sums_dev[device] = static_cast<int*>(p);
    }
    *out = g_sums_dev[device];
    return FG_OK;
}

int grid_for(long long total) {
    return static_cast<int>(std::min<long long>(std::max<long long>((total + 255) / 256, 1), 4096));
}

}  // namespace

using namespace fgrt;

extern "C" fg_status fg_quantized_matmul_noalloc(fg_ctx* ctx, size_t m, size_t n, size_t k,
                                                 const uint8_t* a, uint8_t a_zp, float scale_a,
                                                 const int8_t* b, int8_t b_zp, float scale_b,
                                                 float* c, int accumulate, fg_stream stream) {
    if (!ctx) return set_error(FG_ERR_INVALID, "null context");
    if (m == 0 || n == 0) return FG_OK;
    if (!c || (k > 0 && (!a || !b))) return set_error(FG_ERR_INVALID, "null operand pointer");
    if ((long long)m > kQmmNoAllocMaxM || (long long)n > kQmmNoAllocMaxN)
        return set_error(FG_ERR_UNSUPPORTED,
                         "quantized_matmul_noalloc: m and n must be <= 65536 (the fixed scratch "
                         "holds 65536 row sums and 65536 column sums); got m=" +
                             std::to_string(m) + ", n=" + std::to_string(n));
    if ((long long)k > kQmmNoAllocMaxK)
        return set_error(FG_ERR_UNSUPPORTED,
                         "quantized_matmul_noalloc: k above 65536 would overflow the exact int32 accumulator");
    if (k % 16 || n % 16 || (reinterpret_cast<uintptr_t>(a) & 15) || (reinterpret_cast<uintptr_t>(b) & 15))
        return set_error(FG_ERR_UNSUPPORTED,
                         "quantized_matmul_noalloc: k and n must be multiples of 16 and a, b 16-byte "
                         "aligned (padding the operands would need scratch); use fg_quantized_matmul");
    if (ctx->device < 0 || ctx->device >= kMaxDevices)
        return set_error(FG_ERR_UNSUPPORTED, "quantized_matmul_noalloc: device index above 63");
    FG_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = stream_of(ctx, stream);
    if (k == 0) {  // gemm/mod.rs:509-519: zeros, or C untouched when accumulating
        if (!accumulate) FG_CUDA(cudaMemsetAsync(c, 0, m * n * sizeof(float), st));
        return FG_OK;
    }
    int* sums = nullptr;
    FG_TRY(setup_device(ctx->device, &sums));
    int* row_sum = sums;
    int* col_sum = sums + kQmmNoAllocMaxM;
    const long long M = (long long)m, N = (long long)n, K = (long long)k;
    fg::row_sum_u8_kernel<<<grid_for(M * 32), 256, 0, st>>>(a, M, K, K, row_sum);
    FG_CUDA(cudaMemsetAsync(col_sum, 0, N * sizeof(int), st));
    fg::col_sum_i8_kernel<<<dim3(static_cast<unsigned>((N + 255) / 256), static_cast<unsigned>((K + 255) / 256)),
                            256, 0, st>>>(b, K, N, N, 256, col_sum);
    count_launch(2);
    FG_CUDA(cudaGetLastError());

    fg::TcMaps maps;
    fg::TcArgs args{};
    {
        uint64_t dims[2] = {static_cast<uint64_t>(K), static_cast<uint64_t>(M)};
        uint64_t strides[1] = {static_cast<uint64_t>(K)};
        uint32_t box[2] = {128, 128};
        FG_TRY(encode_map(&maps.a[0], CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, a, dims, strides, box));
    }
    {
        uint64_t dims[2] = {static_cast<uint64_t>(N), static_cast<uint64_t>(K)};
        uint64_t strides[1] = {static_cast<uint64_t>(N)};
        uint32_t box[2] = {128, 128};
        FG_TRY(encode_map(&maps.b[0], CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, b, dims, strides, box));
    }
    args.M = static_cast<int>(M);
    args.N = static_cast<int>(N);
    args.K = static_cast<int>(K);
    args.tiles_m = static_cast<int>((M + 127) / 128);
    args.tiles_n = static_cast<int>((N + CfgQmmNoAlloc::BN - 1) / CfgQmmNoAlloc::BN);
    args.k_blocks = static_cast<int>((K + CfgQmmNoAlloc::BK - 1) / CfgQmmNoAlloc::BK);
    args.batch = 1;
    args.bdims = 1;
    args.bshape[0] = 1;
    args.C = c;
    args.ldc = N;
    args.accumulate = accumulate;
    args.row_sum = row_sum;
    args.col_sum = col_sum;
    args.a_zp = a_zp;
    args.b_zp = b_zp;
    args.scale = scale_a * scale_b;
    args.ops[0] = fg::TcOp{0, 0, 0, 0, 1};  // u8 x s8
    args.status = ctx->d_status;
    args.timeout_ns = 4000000000ull;
    const long long tiles = (long long)args.tiles_m * args.tiles_n;
    const int grid = static_cast<int>(std::min<long long>(tiles, ctx->sm_count));
    fg::tc_gemm_kernel<CfgQmmNoAlloc><<<grid, CfgQmmNoAlloc::THREADS, fg::tc_smem_bytes<CfgQmmNoAlloc>(), st>>>(maps, args);
    count_launch();
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}
