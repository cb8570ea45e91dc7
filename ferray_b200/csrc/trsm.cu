// trsm.cu -- left-side triangular solve op(A) X = alpha B in place on
// device-resident operands (ferray-linalg/src/trsm.rs:46-133).
//
// Structure of the reference, kept: B is scaled by alpha first (trsm.rs:
// 137-153), then the block recursion of trsm.rs:165-200 (lower) and
// trsm.rs:264-300 (upper) splits m at m1 = min(round_up(m / 2, 32), m - 32),
// solves one half, applies the trailing update B2 -= L21 X1 (lower) or
// B1 -= U12 X2 (upper) and solves the other half.  Sub-problems of at most
// 128 rows are one trsm_block_kernel launch that runs the reference's own
// recursion below them (leaves of <= 32 rows, scalar updates) with the
// reference's operation order and roundings, so they are bit-identical to
// the reference.  Above 128 rows the trailing update, which the reference
// runs as a scalar triple loop because its GEMM wants contiguous operands
// (trsm.rs:24-33, 205-225), is one fg_gemm call with alpha = -1, beta = 1
// on the strided sub-blocks, so it gets the tuned kernels (and, in
// FG_MODE_SPLIT, the 3xBF16 / Ozaki forms).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <mutex>

#include "runtime.h"

namespace fgrt {

namespace {

constexpr int kLeaf = 32;  // trsm.rs:33 (NB)

__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double recip_rn(double a) { return __ddiv_rn(1.0, a); }
__device__ __forceinline__ float recip_rn(float a) { return __fdiv_rn(1.0f, a); }

// Diagonal blocks of up to 128 rows run in one launch: the host plans the
// reference's recursion below 128 rows (its split rule, leaves of <= 32
// rows) as a list of operations, and trsm_block_kernel executes them in
// order on a 128 x 32 strip of B staged in shared memory, one thread per
// column.  Every element of B sees the reference's operations in the
// reference's order (b -= a * x as a product, then a difference, the
// update's p ascending; leaves as trsm.rs:227-262 / 304-332), so a block is
// bit-identical to the reference's solve of it.
constexpr int kBlock = 128;    // rows per block launch
constexpr int kCols = 32;      // columns of B per CTA (one warp)
constexpr int kMaxOps = 16;
constexpr int kMaxLeaves = 4;  // m <= 128 splits into at most 4 leaves

struct TrsmOp {
    int leaf;      // 1: solve rows [r0, r0 + rows); 0: update
    int r0, rows;  // rows of B changed
    int s0, k;     // update: B[r0 + i] -= sum_p A[r0 + i][s0 + p] B[s0 + p], p ascending
};
struct TrsmSched {
    int nops, nleaves;
    TrsmOp op[kMaxOps];
};

// Rows [r0, r0 + m) of the block, as trsm.rs:165-200 (lower) / 264-300
// (upper).  A block of m <= 128 rows has at most 4 leaves and 3 updates.
void plan_block(bool upper, int r0, int m, TrsmSched& sc) {
    if (sc.nops >= kMaxOps) {
        sc.nops = kMaxOps + 1;
        return;
    }
    if (m <= kLeaf) {
        if (sc.nleaves >= kMaxLeaves) {
            sc.nops = kMaxOps + 1;
            return;
        }
        sc.op[sc.nops++] = TrsmOp{1, r0, m, r0, 0};
        ++sc.nleaves;
        return;
    }
    const int m1 = std::min((m / 2 + kLeaf - 1) / kLeaf * kLeaf, m - kLeaf);
    const int m2 = m - m1;
    if (!upper) {
        plan_block(upper, r0, m1, sc);
        if (sc.nops < kMaxOps) sc.op[sc.nops++] = TrsmOp{0, r0 + m1, m2, r0, m1};
        plan_block(upper, r0 + m1, m2, sc);
    } else {
        plan_block(upper, r0 + m1, m2, sc);
        if (sc.nops < kMaxOps) sc.op[sc.nops++] = TrsmOp{0, r0, m1, r0 + m1, m2};
        plan_block(upper, r0, m1, sc);
    }
}

constexpr int kThreads = 128;  // 4 warps share one strip: leaves on warp 0, updates on all
constexpr int kAMax = 64;      // an update of a <= 128-row block is at most 64 x 64
constexpr int kAPitch = kAMax + 2;

template <typename T>
struct BlockSmem {
    T xs[kBlock][kCols];            // the strip of B
    T abuf[2][kAMax][kAPitch];      // A operand of the current and the next operation
    T inv[kBlock];                  // 1 / a_ii of the current leaf
};

// Global -> shared copy of one element (cp.async, no register staging);
// `valid` false writes zero.
template <typename T>
__device__ __forceinline__ void cp_async_elem(T* smem, const T* gmem, bool valid) {
    const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(s), "l"(gmem), "n"(sizeof(T)),
                 "r"(valid ? static_cast<int>(sizeof(T)) : 0)
                 : "memory");
}

// Issue the copies of operation op's A block into buf: a leaf's triangle
// A[r0.., r0..] (rows x rows) or an update's A[r0.., s0..] (rows x k).
template <typename T>
__device__ __forceinline__ void stage_op(T (*buf)[kAPitch], const TrsmOp& op, const T* __restrict__ a, long long lda) {
    const int cols = op.leaf ? op.rows : op.k;
    const int c0 = op.leaf ? op.r0 : op.s0;
    const int total = op.rows * cols;
    for (int e = threadIdx.x; e < total; e += kThreads) {
        const int i = e / cols, c = e - i * cols;
        cp_async_elem(&buf[i][c], a + (op.r0 + i) * lda + c0 + c, true);
    }
}

// Leaf (warp 0): rows [r0, r0 + m) of the strip, one column per lane, the
// triangle in tri (trsm.rs:227-262 lower, 304-332 upper).
template <typename T, bool UPPER>
__device__ __forceinline__ void block_leaf(BlockSmem<T>& sm, const T (*tri)[kAPitch], int r0, int m,
                                           int unit_diag) {
    const int lane = threadIdx.x;
    if (!unit_diag && lane < m) sm.inv[lane] = recip_rn(tri[lane][lane]);
    __syncwarp();
    T x[kLeaf];
#pragma unroll
    for (int i = 0; i < kLeaf; ++i) x[i] = i < m ? sm.xs[r0 + i][lane] : T(0);
    if constexpr (!UPPER) {
#pragma unroll
        for (int i = 0; i < kLeaf; ++i) {
            if (i < m) {
                T v = x[i];
#pragma unroll
                for (int p = 0; p < i; ++p) v = sub_rn(v, mul_rn(tri[i][p], x[p]));
                if (!unit_diag) v = mul_rn(v, sm.inv[i]);
                x[i] = v;
            }
        }
    } else {
#pragma unroll
        for (int i = kLeaf - 1; i >= 0; --i) {
            if (i < m) {
                T v = x[i];
#pragma unroll
                for (int p = i + 1; p < kLeaf; ++p)
                    if (p < m) v = sub_rn(v, mul_rn(tri[i][p], x[p]));
                if (!unit_diag) v = mul_rn(v, sm.inv[i]);
                x[i] = v;
            }
        }
    }
#pragma unroll
    for (int i = 0; i < kLeaf; ++i)
        if (i < m) sm.xs[r0 + i][lane] = x[i];
}

// B[r0 + i] -= sum_p A[r0 + i][s0 + p] B[s0 + p] for i < rows, p ascending
// (trsm.rs:205-225); A[r0 + i][s0 + p] = blk[i][p].  Warp w takes the
// 8-row chunks w, w + 4, ... (independent chains per chunk).
template <typename T>
__device__ __forceinline__ void block_update(BlockSmem<T>& sm, const T (*blk)[kAPitch], int r0, int rows, int s0,
                                             int k) {
    const int lane = threadIdx.x % 32, warp = threadIdx.x / 32;
    for (int i0 = warp * 8; i0 < rows; i0 += 32) {
        T acc[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) acc[u] = i0 + u < rows ? sm.xs[r0 + i0 + u][lane] : T(0);
#pragma unroll 4
        for (int p = 0; p < k; ++p) {
            const T xp = sm.xs[s0 + p][lane];
#pragma unroll
            for (int u = 0; u < 8; ++u) acc[u] = sub_rn(acc[u], mul_rn(blk[i0 + u][p], xp));
        }
#pragma unroll
        for (int u = 0; u < 8; ++u)
            if (i0 + u < rows) sm.xs[r0 + i0 + u][lane] = acc[u];
    }
}

// One diagonal block of m <= 128 rows (a, b at its top-left corner); a CTA
// holds a 32-column strip of B.  Each operation's A block is copied into
// shared memory (cp.async) while the previous operation runs.
template <typename T, bool UPPER>
__global__ void __launch_bounds__(kThreads) trsm_block_kernel(const __grid_constant__ TrsmSched sc, int m,
                                                              long long n, const T* __restrict__ a, long long lda,
                                                              T* __restrict__ b, long long ldb, int unit_diag) {
    extern __shared__ __align__(16) unsigned char trsm_smem[];
    BlockSmem<T>& sm = *reinterpret_cast<BlockSmem<T>*>(trsm_smem);
    const int lane = threadIdx.x % 32, warp = threadIdx.x / 32;
    const long long j = blockIdx.x * (long long)kCols + lane;
    const bool live = j < n;
    for (int r = warp; r < m; r += kThreads / 32) cp_async_elem(&sm.xs[r][lane], live ? b + r * ldb + j : b, live);
    stage_op(sm.abuf[0], sc.op[0], a, lda);
    asm volatile("cp.async.commit_group;" ::: "memory");
    for (int o = 0; o < sc.nops; ++o) {
        if (o + 1 < sc.nops) {
            stage_op(sm.abuf[(o + 1) & 1], sc.op[o + 1], a, lda);
            asm volatile("cp.async.commit_group;" ::: "memory");
            asm volatile("cp.async.wait_group 1;" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        }
        __syncthreads();  // op o's A block and every earlier write to the strip are visible
        const TrsmOp op = sc.op[o];
        if (op.leaf) {
            if (warp == 0) block_leaf<T, UPPER>(sm, sm.abuf[o & 1], op.r0, op.rows, unit_diag);
        } else {
            block_update<T>(sm, sm.abuf[o & 1], op.r0, op.rows, op.s0, op.k);
        }
        __syncthreads();  // buffer o & 1 is refilled at o + 1
    }
    if (live)
        for (int r = warp; r < m; r += kThreads / 32) b[r * ldb + j] = sm.xs[r][lane];
}

// B *= alpha over an m x n block with row stride ldb.
template <typename T>
__global__ void trsm_scale_kernel(long long m, long long n, T alpha, T* __restrict__ b, long long ldb) {
    const long long total = m * n;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long i = e / n, j = e - i * n;
        b[i * ldb + j] = mul_rn(b[i * ldb + j], alpha);
    }
}

// Smallest rows, k and n of an f64 trailing update that runs the Ozaki
// split form in FG_MODE_SPLIT.
static long long ozaki_min() {
    static long long v = [] {
        const char* e = getenv("FG_TRSM_OZAKI_MIN");
        return e ? atoll(e) : 4096LL;
    }();
    return v;
}

template <typename T>
struct Trsm {
    fg_ctx* ctx;
    fg_dtype dtype;
    fg_mode mode;
    bool upper;
    int unit;
    long long n, lda, ldb;
    cudaStream_t st;

    fg_status block(long long m, const T* a, T* b) {
        TrsmSched sc{};
        plan_block(upper, 0, static_cast<int>(m), sc);
        if (sc.nops > kMaxOps) return set_error(FG_ERR_INVALID, "trsm: block plan overflow");
        for (int o = 0; o < sc.nops; ++o)
            if (sc.op[o].rows > kAMax || (!sc.op[o].leaf && sc.op[o].k > kAMax))
                return set_error(FG_ERR_INVALID, "trsm: block plan exceeds the staging buffer");
        const unsigned grid = static_cast<unsigned>((n + kCols - 1) / kCols);
        constexpr int smem = static_cast<int>(sizeof(BlockSmem<T>));
        auto kern = upper ? trsm_block_kernel<T, true> : trsm_block_kernel<T, false>;
        static std::once_flag once;
        static cudaError_t attr_err = cudaSuccess;
        std::call_once(once, [] {
            for (auto k : {trsm_block_kernel<T, true>, trsm_block_kernel<T, false>}) {
                const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
                if (e != cudaSuccess) attr_err = e;
            }
        });
        FG_CUDA(attr_err);
        ProfScope prof("trsm_block", st);
        kern<<<grid, kThreads, smem, st>>>(sc, static_cast<int>(m), n, a, lda, b, ldb, unit);
        count_launch();
        FG_CUDA(cudaGetLastError());
        return FG_OK;
    }

    // c (rows x n) -= a (rows x k, stride lda) * x (k x n, stride ldb).  In
    // split mode an f64 update smaller than ozaki_min() in rows, k or n runs
    // plain: the Ozaki form's slicing passes cost more than they save there
    // (measured on B200: at 8192^2 a floor of 4096 gave 19.8 ms, 2048 20.1,
    // 1024 21.8, none 44.8), and the solve's residual is set by the
    // substitution, not by these updates.
    fg_status update(long long rows, long long k, const T* a, const T* x, T* c) {
        const T minus_one = T(-1), one = T(1);
        fg_mode md = mode;
        if (dtype == FG_F64 && mode != FG_MODE_PLAIN && (rows < ozaki_min() || k < ozaki_min() || n < ozaki_min()))
            md = FG_MODE_PLAIN;
        return fg_gemm(ctx, dtype, md, 0, static_cast<size_t>(rows), static_cast<size_t>(n),
                       static_cast<size_t>(k), &minus_one, a, static_cast<size_t>(lda), x,
                       static_cast<size_t>(ldb), &one, c, static_cast<size_t>(ldb), 0, st);
    }

    fg_status solve(long long m, const T* a, T* b) {
        if (m <= kBlock) return block(m, a, b);
        const long long m1 = std::min<long long>((m / 2 + kLeaf - 1) / kLeaf * kLeaf, m - kLeaf);
        const long long m2 = m - m1;
        const T* a22 = a + m1 * lda + m1;
        T* b2 = b + m1 * ldb;
        if (!upper) {
            FG_TRY(solve(m1, a, b));                    // L11 X1 = B1
            FG_TRY(update(m2, m1, a + m1 * lda, b, b2));  // B2 -= L21 X1
            return solve(m2, a22, b2);                  // L22 X2 = B2
        }
        FG_TRY(solve(m2, a22, b2));              // U22 X2 = B2
        FG_TRY(update(m1, m2, a + m1, b2, b));   // B1 -= U12 X2
        return solve(m1, a, b);                  // U11 X1 = B1
    }
};

template <typename T>
fg_status run_trsm(fg_ctx* ctx, fg_dtype dtype, fg_mode mode, int upper, int unit_diag, long long m, long long n,
                   const void* alpha, const void* a, long long lda, void* b, long long ldb, cudaStream_t st) {
    const T al = alpha ? *static_cast<const T*>(alpha) : T(1);
    T* bb = static_cast<T*>(b);
    if (al != T(1)) {
        const long long total = m * n;
        const int grid = static_cast<int>(std::min<long long>((total + 255) / 256, 4096));
        trsm_scale_kernel<T><<<grid, 256, 0, st>>>(m, n, al, bb, ldb);
        count_launch();
        FG_CUDA(cudaGetLastError());
    }
    Trsm<T> t{ctx, dtype, mode, upper != 0, unit_diag ? 1 : 0, n, lda, ldb, st};
    return t.solve(m, static_cast<const T*>(a), bb);
}

}  // namespace

}  // namespace fgrt

using namespace fgrt;

extern "C" {

fg_status fg_trsm_left(fg_ctx* ctx, fg_dtype dtype, fg_mode mode, int upper, int unit_diag, size_t m, size_t n,
                       const void* alpha, const void* a, size_t lda, void* b, size_t ldb, fg_stream stream) {
    if (!ctx) return set_error(FG_ERR_INVALID, "trsm: null context");
    if (dtype != FG_F64 && dtype != FG_F32)
        return set_error(FG_ERR_DTYPE, "trsm: f64 and f32 only (trsm.rs has no other element types)");
    if (mode != FG_MODE_PLAIN && mode != FG_MODE_SPLIT && mode != FG_MODE_SPLIT_F16)
        return set_error(FG_ERR_INVALID, "trsm: bad mode");
    if (m == 0 || n == 0) return FG_OK;  // trsm.rs:56-58: nothing to do, B untouched
    if (!a || !b) return set_error(FG_ERR_INVALID, "trsm: null operand");
    if (lda < m || ldb < n)
        return set_error(FG_ERR_SHAPE, "trsm: lda must be >= m and ldb >= n");
    if (m > (1ull << 31) || n > (1ull << 36)) return set_error(FG_ERR_SHAPE, "trsm: dimensions too large");
    const cudaStream_t st = stream_of(ctx, stream);
    const long long M = static_cast<long long>(m), N = static_cast<long long>(n);
    if (dtype == FG_F64)
        return run_trsm<double>(ctx, dtype, mode, upper, unit_diag, M, N, alpha, a, static_cast<long long>(lda), b,
                                static_cast<long long>(ldb), st);
    return run_trsm<float>(ctx, dtype, mode, upper, unit_diag, M, N, alpha, a, static_cast<long long>(lda), b,
                           static_cast<long long>(ldb), st);
}

}  // extern "C"
