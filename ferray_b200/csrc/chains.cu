// chains.cu -- GEMM-heavy callers of matmul run natively on device-resident
// operands: multi_dot (products/mod.rs:776-902) and matrix_power
// (solve.rs:456-494).  Intermediates stay in HBM (stream-ordered scratch);
// every product is one fg_gemm call, so it gets the tuned kernels.
#include <cuda_runtime.h>

#include <cstring>
#include <vector>

#include "prep_kernels.cuh"
#include "runtime.h"

namespace fgrt {

namespace {

bool chain_dtype_ok(fg_dtype d) { return d == FG_F64 || d == FG_F32 || d == FG_C64 || d == FG_C32; }

// Optimal parenthesisation by the O(n^3) chain-order dynamic programme of
// products/mod.rs:839-855: cost[i][j] = min over k of cost[i][k] +
// cost[k+1][j] + d_i d_{k+1} d_{j+1} (u64), the first k reaching the minimum
// wins.  split is n x n row-major.
void chain_order(size_t n, const int64_t* dims, std::vector<size_t>& split) {
    std::vector<uint64_t> cost(n * n, 0);
    split.assign(n * n, 0);
    for (size_t len = 2; len <= n; ++len) {
        for (size_t i = 0; i + len <= n; ++i) {
            const size_t j = i + len - 1;
            cost[i * n + j] = UINT64_MAX;
            for (size_t k = i; k < j; ++k) {
                const uint64_t q = cost[i * n + k] + cost[(k + 1) * n + j] +
                                   static_cast<uint64_t>(dims[i]) * static_cast<uint64_t>(dims[k + 1]) *
                                       static_cast<uint64_t>(dims[j + 1]);
                if (q < cost[i * n + j]) {
                    cost[i * n + j] = q;
                    split[i * n + j] = k;
                }
            }
        }
    }
}

struct ChainRun {
    fg_ctx* ctx;
    fg_dtype dtype;
    fg_mode mode;
    size_t n;
    const void* const* mats;
    const int64_t* dims;
    const std::vector<size_t>* split;
    cudaStream_t st;
    std::vector<Scratch*> owned;  // intermediates, freed (stream-ordered) at the end
    ~ChainRun() {
        for (Scratch* s : owned) delete s;
    }

    // Product of matrices i..j into dst (dims[i] x dims[j+1]); dst may be
    // null: then an intermediate is allocated and returned.
    fg_status product(size_t i, size_t j, void* dst, const void** out) {
        if (i == j) {
            *out = mats[i];
            return FG_OK;
        }
        const size_t k = (*split)[i * n + j];
        const void *left, *right;
        FG_TRY(product(i, k, nullptr, &left));
        FG_TRY(product(k + 1, j, nullptr, &right));
        const size_t m = static_cast<size_t>(dims[i]), kk = static_cast<size_t>(dims[k + 1]),
                     nn = static_cast<size_t>(dims[j + 1]);
        if (!dst) {
            Scratch* s = new Scratch();
            owned.push_back(s);
            FG_TRY(s->alloc(m * nn * out_size(dtype), st));
            dst = s->p;
        }
        FG_TRY(fg_gemm(ctx, dtype, mode, 0, m, nn, kk, nullptr, left, kk, right, nn, nullptr, dst, nn, 0, st));
        *out = dst;
        return FG_OK;
    }
};

// out (n x n, contiguous) = I: zero fill, then 1 on the diagonal (real part
// for complex; `vals` values per element, `step` = (n + 1) * vals).
template <typename T>
__global__ void diag_one_kernel(T* __restrict__ out, long long n, long long step) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i * step] = T(1);
}

fg_status write_identity(fg_dtype d, void* out, long long n, cudaStream_t st) {
    FG_CUDA(cudaMemsetAsync(out, 0, static_cast<size_t>(n * n) * out_size(d), st));
    const int grid = static_cast<int>(std::min<long long>((n + 255) / 256, 1024));
    const long long vals = is_complex(d) ? 2 : 1;
    if (d == FG_F64 || d == FG_C64)
        diag_one_kernel<double><<<grid, 256, 0, st>>>(static_cast<double*>(out), n, (n + 1) * vals);
    else
        diag_one_kernel<float><<<grid, 256, 0, st>>>(static_cast<float*>(out), n, (n + 1) * vals);
    count_launch();
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

}  // namespace

}  // namespace fgrt

using namespace fgrt;

extern "C" {

fg_status fg_multi_dot_order(size_t count, const int64_t* dims, size_t* split) {
    if (count < 2 || !dims || !split) return set_error(FG_ERR_INVALID, "multi_dot: need at least 2 matrices");
    for (size_t i = 0; i <= count; ++i)
        if (dims[i] < 0) return set_error(FG_ERR_SHAPE, "multi_dot: negative dimension");
    std::vector<size_t> sp;
    chain_order(count, dims, sp);
    std::memcpy(split, sp.data(), sp.size() * sizeof(size_t));
    return FG_OK;
}

fg_status fg_multi_dot(fg_ctx* ctx, fg_dtype dtype, fg_mode mode, size_t count, const void* const* mats,
                       const int64_t* dims, void* out, fg_stream stream) {
    if (!ctx) return set_error(FG_ERR_INVALID, "null context");
    if (!chain_dtype_ok(dtype)) return set_error(FG_ERR_DTYPE, "multi_dot: dtype must be f64, f32, c64 or c32");
    if (count < 2 || !mats || !dims || !out) return set_error(FG_ERR_INVALID, "multi_dot: need at least 2 matrices");
    for (size_t i = 0; i <= count; ++i)
        if (dims[i] <= 0) return set_error(FG_ERR_SHAPE, "multi_dot: dimensions must be positive");
    for (size_t i = 0; i < count; ++i)
        if (!mats[i]) return set_error(FG_ERR_INVALID, "multi_dot: null matrix pointer");
    FG_CUDA(cudaSetDevice(ctx->device));
    std::vector<size_t> split;
    chain_order(count, dims, split);
    ChainRun run{ctx, dtype, mode, count, mats, dims, &split, stream_of(ctx, stream), {}};
    const void* res = nullptr;
    return run.product(0, count - 1, out, &res);
}

fg_status fg_matrix_power(fg_ctx* ctx, fg_dtype dtype, fg_mode mode, size_t n, const void* a,
                          int64_t exponent, void* out, fg_stream stream) {
    if (!ctx) return set_error(FG_ERR_INVALID, "null context");
    if (!chain_dtype_ok(dtype)) return set_error(FG_ERR_DTYPE, "matrix_power: dtype must be f64, f32, c64 or c32");
    if (!out || (n > 0 && !a)) return set_error(FG_ERR_INVALID, "matrix_power: null pointer");
    if (exponent < 0)
        return set_error(FG_ERR_UNSUPPORTED, "matrix_power: negative powers need inv(A), which is not on this path");
    FG_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = stream_of(ctx, stream);
    if (n == 0) return FG_OK;
    const size_t bytes = n * n * out_size(dtype);
    if (exponent == 0) return write_identity(dtype, out, static_cast<long long>(n), st);
    // Exponentiation by squaring in the order of solve.rs:480-491: result
    // starts at I, result = result @ base on a set bit, base = base @ base
    // while bits remain (the squaring after the last bit is not needed for
    // the result and is skipped).  Buffers: result ping-pongs between `out`
    // and one scratch; base between two scratch buffers (base starts as A).
    Scratch s_res, s_b0, s_b1;
    FG_TRY(s_res.alloc(bytes, st));
    FG_TRY(s_b0.alloc(bytes, st));
    FG_TRY(s_b1.alloc(bytes, st));
    void* res_bufs[2] = {out, s_res.p};
    int ri = 0;
    FG_TRY(write_identity(dtype, res_bufs[ri], static_cast<long long>(n), st));
    const void* base = a;
    void* base_bufs[2] = {s_b0.p, s_b1.p};
    int bi = 0;
    uint64_t p = static_cast<uint64_t>(exponent);
    while (p > 0) {
        if (p & 1) {
            FG_TRY(fg_gemm(ctx, dtype, mode, 0, n, n, n, nullptr, res_bufs[ri], n, base, n, nullptr,
                           res_bufs[ri ^ 1], n, 0, st));
            ri ^= 1;
        }
        p >>= 1;
        if (p > 0) {
            FG_TRY(fg_gemm(ctx, dtype, mode, 0, n, n, n, nullptr, base, n, base, n, nullptr, base_bufs[bi], n,
                           0, st));
            base = base_bufs[bi];
            bi ^= 1;
        }
    }
    if (res_bufs[ri] != out) FG_CUDA(cudaMemcpyAsync(out, res_bufs[ri], bytes, cudaMemcpyDeviceToDevice, st));
    return FG_OK;
}

}  // extern "C"
