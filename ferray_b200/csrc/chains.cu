// chains.cu -- GEMM-heavy callers of matmul run natively on device-resident
// operands: multi_dot (products/mod.rs:776-902) and matrix_power
// (solve.rs:456-494).  Intermediates stay in HBM (stream-ordered scratch);
// every product is one fg_gemm call, so it gets the tuned kernels.
#include <cuda_runtime.h>

#include <cstring>
#include <string>
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

// N-D permutation (up to 8 dims) of a contiguous row-major array into a
// contiguous one: out[o] = in[sum_d idx_d(o) * in_stride[perm[d]]], elements
// of E bytes moved as 4- or 8-byte words.
struct PermuteArgs {
    int nd;
    long long out_shape[8];
    long long in_stride[8];  // elements, of the input axis that is output axis d
};

template <typename W, int WPE>
__global__ void permute_kernel(const W* __restrict__ in, W* __restrict__ out, long long total,
                               PermuteArgs pa) {
    for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < total;
         o += (long long)gridDim.x * blockDim.x) {
        long long rem = o, src = 0;
#pragma unroll
        for (int d = 7; d >= 0; --d) {
            if (d < pa.nd) {
                const long long idx = rem % pa.out_shape[d];
                rem /= pa.out_shape[d];
                src += idx * pa.in_stride[d];
            }
        }
#pragma unroll
        for (int w = 0; w < WPE; ++w) out[o * WPE + w] = in[src * WPE + w];
    }
}

// Permutes `in` (shape, nd) by perm into `out`; no-op (returns in) for the
// identity permutation.
fg_status permute(fg_dtype d, const void* in, int nd, const int64_t* shape, const int* perm, Scratch& sc,
                  const void** result, cudaStream_t st) {
    bool ident = true;
    for (int i = 0; i < nd; ++i) ident = ident && perm[i] == i;
    if (ident) {
        *result = in;
        return FG_OK;
    }
    PermuteArgs pa{};
    pa.nd = nd;
    long long stride[8], total = 1;
    for (int i = nd - 1; i >= 0; --i) {
        stride[i] = total;
        total *= shape[i];
    }
    for (int i = 0; i < nd; ++i) {
        pa.out_shape[i] = shape[perm[i]];
        pa.in_stride[i] = stride[perm[i]];
    }
    const size_t es = out_size(d);
    FG_TRY(sc.alloc(static_cast<size_t>(std::max<long long>(total, 1)) * es, st));
    const int grid = static_cast<int>(std::min<long long>(std::max<long long>((total + 255) / 256, 1), 8192));
    using U64 = unsigned long long;
    if (es == 4)
        permute_kernel<uint32_t, 1><<<grid, 256, 0, st>>>(static_cast<const uint32_t*>(in),
                                                          static_cast<uint32_t*>(sc.p), total, pa);
    else if (es == 8)
        permute_kernel<U64, 1><<<grid, 256, 0, st>>>(static_cast<const U64*>(in), static_cast<U64*>(sc.p),
                                                     total, pa);
    else
        permute_kernel<U64, 2><<<grid, 256, 0, st>>>(static_cast<const U64*>(in), static_cast<U64*>(sc.p),
                                                     total, pa);
    count_launch();
    FG_CUDA(cudaGetLastError());
    *result = sc.p;
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

fg_status fg_tensordot(fg_ctx* ctx, fg_dtype dtype, fg_mode mode, const void* a, int ndim_a,
                       const int64_t* shape_a, const void* b, int ndim_b, const int64_t* shape_b, int naxes,
                       const int* axes_a, const int* axes_b, void* out, int64_t* out_shape, int* out_ndim,
                       fg_stream stream) {
    if (!ctx) return set_error(FG_ERR_INVALID, "null context");
    if (!chain_dtype_ok(dtype)) return set_error(FG_ERR_DTYPE, "tensordot: dtype must be f64, f32, c64 or c32");
    if (ndim_a < 0 || ndim_b < 0 || ndim_a > 8 || ndim_b > 8 || naxes < 0 || !out_shape || !out_ndim)
        return set_error(FG_ERR_INVALID, "tensordot: bad ranks or null output arguments");
    if (naxes > 0 && (!axes_a || !axes_b)) return set_error(FG_ERR_INVALID, "tensordot: null axes");
    // checks and free axes as products/tensordot.rs:67-97
    for (int i = 0; i < naxes; ++i) {
        if (axes_a[i] < 0 || axes_a[i] >= ndim_a || axes_b[i] < 0 || axes_b[i] >= ndim_b)
            return set_error(FG_ERR_SHAPE, "tensordot: axis out of bounds");
        if (shape_a[axes_a[i]] != shape_b[axes_b[i]])
            return set_error(FG_ERR_SHAPE, "tensordot: contracted dimensions must match");
        for (int j = 0; j < i; ++j)
            if (axes_a[j] == axes_a[i] || axes_b[j] == axes_b[i])
                return set_error(FG_ERR_SHAPE, "tensordot: repeated axis");
    }
    auto contains = [](const int* ax, int n, int v) {
        for (int i = 0; i < n; ++i)
            if (ax[i] == v) return true;
        return false;
    };
    int perm_a[8], perm_b[8], nfa = 0, nfb = 0;
    long long free_a = 1, free_b = 1, contract = 1;
    int nout = 0;
    for (int i = 0; i < ndim_a; ++i)
        if (!contains(axes_a, naxes, i)) {
            perm_a[nfa++] = i;
            free_a *= shape_a[i];
            out_shape[nout++] = shape_a[i];
        }
    for (int i = 0; i < naxes; ++i) {
        perm_a[nfa + i] = axes_a[i];
        contract *= shape_a[axes_a[i]];
    }
    for (int i = 0; i < naxes; ++i) perm_b[i] = axes_b[i];
    for (int i = 0; i < ndim_b; ++i)
        if (!contains(axes_b, naxes, i)) {
            perm_b[naxes + nfb++] = i;
            free_b *= shape_b[i];
            out_shape[nout++] = shape_b[i];
        }
    *out_ndim = nout;
    FG_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = stream_of(ctx, stream);
    if (free_a == 0 || free_b == 0) return FG_OK;
    if (!a || !b || !out) return set_error(FG_ERR_INVALID, "tensordot: null pointer");
    Scratch sa, sb;
    const void *pa = a, *pb = b;
    FG_TRY(permute(dtype, a, ndim_a, shape_a, perm_a, sa, &pa, st));
    FG_TRY(permute(dtype, b, ndim_b, shape_b, perm_b, sb, &pb, st));
    // (free_a x contract) @ (contract x free_b); contract == 1 with no axes
    // is the outer product
    return fg_gemm(ctx, dtype, mode, 0, static_cast<size_t>(free_a), static_cast<size_t>(free_b),
                   static_cast<size_t>(contract), nullptr, pa, static_cast<size_t>(contract), pb,
                   static_cast<size_t>(free_b), nullptr, out, static_cast<size_t>(free_b), 0, st);
}

// Two-operand einsum "ab..,cd..->xy.." (labels a-z, A-Z; implicit output =
// the labels that appear once, sorted, as numpy does).  Labels split into
// batch (in both operands and the output), free-a, free-b (one operand and
// the output) and contracted (both operands, not the output; a label in one
// operand only and not in the output is summed by contracting with ones,
// which is not supported here).  A is permuted to [batch, free_a, contract],
// B to [batch, contract, free_b], one batched GEMM forms
// [batch, free_a, free_b], and a last permute puts the output in the
// requested label order.  This covers the reference's matmul shortcut
// (products/einsum/mod.rs:251-282) and every other pairwise contraction
// without repeated labels inside one operand.
fg_status fg_einsum(fg_ctx* ctx, fg_dtype dtype, fg_mode mode, const char* subscripts, const void* a, int ndim_a,
                    const int64_t* shape_a, const void* b, int ndim_b, const int64_t* shape_b, void* out,
                    int64_t* out_shape, int* out_ndim, fg_stream stream) {
    if (!ctx || !subscripts || !out_shape || !out_ndim) return set_error(FG_ERR_INVALID, "einsum: null argument");
    if (!chain_dtype_ok(dtype)) return set_error(FG_ERR_DTYPE, "einsum: dtype must be f64, f32, c64 or c32");
    std::string spec;
    for (const char* c = subscripts; *c; ++c)
        if (*c != ' ') spec.push_back(*c);
    const size_t comma = spec.find(','), arrow = spec.find("->");
    if (comma == std::string::npos || spec.find(',', comma + 1) != std::string::npos ||
        (arrow != std::string::npos && arrow < comma))
        return set_error(FG_ERR_INVALID, "einsum: expected exactly two operands 'ab,bc->ac'");
    const std::string la = spec.substr(0, comma);
    const std::string lb = spec.substr(comma + 1, arrow == std::string::npos ? std::string::npos : arrow - comma - 1);
    auto is_label = [](char c) { return (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z'); };
    for (char c : la + lb)
        if (!is_label(c)) return set_error(FG_ERR_UNSUPPORTED, "einsum: only letter labels (no ellipsis)");
    if ((int)la.size() != ndim_a || (int)lb.size() != ndim_b)
        return set_error(FG_ERR_SHAPE, "einsum: subscripts do not match the operand ranks");
    for (size_t i = 0; i < la.size(); ++i)
        if (la.find(la[i]) != i) return set_error(FG_ERR_UNSUPPORTED, "einsum: repeated label within an operand");
    for (size_t i = 0; i < lb.size(); ++i)
        if (lb.find(lb[i]) != i) return set_error(FG_ERR_UNSUPPORTED, "einsum: repeated label within an operand");
    std::string lo;
    if (arrow != std::string::npos) {
        lo = spec.substr(arrow + 2);
        for (size_t i = 0; i < lo.size(); ++i) {
            if (!is_label(lo[i]) || lo.find(lo[i]) != i) return set_error(FG_ERR_INVALID, "einsum: bad output labels");
            if (la.find(lo[i]) == std::string::npos && lb.find(lo[i]) == std::string::npos)
                return set_error(FG_ERR_INVALID, "einsum: output label not in any operand");
        }
    } else {
        for (char c = 'A'; c <= 'z'; ++c) {
            if (!is_label(c)) continue;
            const int n = (la.find(c) != std::string::npos) + (lb.find(c) != std::string::npos);
            if (n == 1) lo.push_back(c);
        }
    }
    if (lo.size() > 8 || la.size() > 8 || lb.size() > 8) return set_error(FG_ERR_UNSUPPORTED, "einsum: more than 8 dims");
    auto size_of = [&](char c, int64_t* v) -> bool {
        const size_t ia = la.find(c), ib = lb.find(c);
        if (ia != std::string::npos && ib != std::string::npos && shape_a[ia] != shape_b[ib]) return false;
        *v = ia != std::string::npos ? shape_a[ia] : shape_b[ib];
        return true;
    };
    std::string batch, fa, fb, con;
    for (char c : la) {
        const bool inb = lb.find(c) != std::string::npos, ino = lo.find(c) != std::string::npos;
        if (inb && ino) batch.push_back(c);
        else if (inb) con.push_back(c);
        else if (ino) fa.push_back(c);
        else return set_error(FG_ERR_UNSUPPORTED, "einsum: label summed within one operand");
    }
    for (char c : lb) {
        const bool ina = la.find(c) != std::string::npos, ino = lo.find(c) != std::string::npos;
        if (!ina && ino) fb.push_back(c);
        else if (!ina) return set_error(FG_ERR_UNSUPPORTED, "einsum: label summed within one operand");
    }
    int64_t nb = 1, m = 1, n = 1, k = 1, v;
    for (char c : batch) { if (!size_of(c, &v)) return set_error(FG_ERR_SHAPE, "einsum: dimension mismatch"); nb *= v; }
    for (char c : fa) { size_of(c, &v); m *= v; }
    for (char c : fb) { size_of(c, &v); n *= v; }
    for (char c : con) { if (!size_of(c, &v)) return set_error(FG_ERR_SHAPE, "einsum: dimension mismatch"); k *= v; }
    *out_ndim = static_cast<int>(lo.size());
    for (size_t i = 0; i < lo.size(); ++i) size_of(lo[i], &out_shape[i]);
    FG_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = stream_of(ctx, stream);
    if (nb * m * n == 0) return FG_OK;
    if (!a || !b || !out) return set_error(FG_ERR_INVALID, "einsum: null pointer");
    int perm_a[8], perm_b[8], perm_o[8];
    const std::string oa = batch + fa + con, ob = batch + con + fb, om = batch + fa + fb;
    for (size_t i = 0; i < oa.size(); ++i) perm_a[i] = static_cast<int>(la.find(oa[i]));
    for (size_t i = 0; i < ob.size(); ++i) perm_b[i] = static_cast<int>(lb.find(ob[i]));
    Scratch sa, sb, sm;
    const void *pa, *pb;
    FG_TRY(permute(dtype, a, ndim_a, shape_a, perm_a, sa, &pa, st));
    FG_TRY(permute(dtype, b, ndim_b, shape_b, perm_b, sb, &pb, st));
    // [batch, free_a, free_b] -> requested order; identity writes straight to out
    int64_t mshape[8];
    for (size_t i = 0; i < om.size(); ++i) size_of(om[i], &mshape[i]);
    for (size_t i = 0; i < lo.size(); ++i) perm_o[i] = static_cast<int>(om.find(lo[i]));
    bool ident = true;
    for (size_t i = 0; i < lo.size(); ++i) ident = ident && perm_o[i] == static_cast<int>(i);
    void* dst = out;
    if (!ident) {
        FG_TRY(sm.alloc(static_cast<size_t>(nb * m * n) * out_size(dtype), st));
        dst = sm.p;
    }
    FG_TRY(fg_gemm_batched_strided(ctx, dtype, mode, 0, static_cast<size_t>(nb), static_cast<size_t>(m),
                                   static_cast<size_t>(n), static_cast<size_t>(k), nullptr, pa,
                                   static_cast<size_t>(k), m * k, pb, static_cast<size_t>(n), k * n, nullptr, dst,
                                   static_cast<size_t>(n), m * n, 0, st));
    if (!ident) {
        Scratch tmp;
        const void* res = nullptr;
        FG_TRY(permute(dtype, dst, static_cast<int>(om.size()), mshape, perm_o, tmp, &res, st));
        FG_CUDA(cudaMemcpyAsync(out, res, static_cast<size_t>(nb * m * n) * out_size(dtype),
                                cudaMemcpyDeviceToDevice, st));
    }
    return FG_OK;
}

}  // extern "C"
