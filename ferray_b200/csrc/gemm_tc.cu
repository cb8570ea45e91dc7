// gemm_tc.cu -- host launchers of the tcgen05 GEMM family:
//   * i8 x i8 and u8 x i8 -> i32 (exact, wrapping)            [kind::i8]
//   * i16 x i16 -> i32 as 4 byte-slice products, recombined    [kind::i8]
//   * quantized u8 x i8 -> f32 with the zero-point correction
//     fused into the epilogue                                  [kind::i8]
//   * 3xBF16 SGEMM / CGEMM (split mode)                        [kind::f16]
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdlib>
#include <vector>

#include "prep_kernels.cuh"
#include "runtime.h"
#include "tc_gemm.cuh"
#include "tc_gemm2.cuh"
#include "tune.h"

namespace fgrt {

using namespace fg;

// i8 variants (tuned): 128 x 256 tiles, 4 stages; 128 x 128 tiles,
// 6 stages, for problems with few output tiles.
using CfgI8 = TcCfg<KIND_I8, 256, 4, 1, 1, 1, 1, EPI_I32>;
using CfgI8n128 = TcCfg<KIND_I8, 128, 6, 1, 1, 1, 1, EPI_I32>;
// 256 x 256 tiles on CTA pairs (cta_group::2), 6 stages of 32 KB per CTA.
using CfgI8Pair = Tc2Cfg<KIND_I8, 256, 7, 1, 1, 1, 1, EPI_I32>;
// 256 x 512 tiles on CTA pairs: one A tile feeds two N = 256 MMAs into two
// TMEM accumulators (all 512 columns, single-buffered); 4 stages of 48 KB.
using CfgI8PairW = Tc2Cfg<KIND_I8, 256, 4, 1, 2, 2, 2, EPI_I32, 0, 1>;
using CfgQmm = TcCfg<KIND_I8, 256, 4, 1, 1, 1, 1, EPI_QMM>;
using CfgQmmPair = Tc2Cfg<KIND_I8, 256, 6, 1, 1, 1, 1, EPI_QMM>;
using CfgI16 = TcCfg<KIND_I8, 128, 3, 2, 2, 3, 4, EPI_I16>;
// 3 products: one accumulator (the 2-slice representation error, about
// 2^-18 |a||b| per product, dominates whatever the accumulation does).
// 6 products: accumulator 0 holds hi*hi, accumulator 1 the corrections.
using CfgBf16x3 = TcCfg<KIND_BF16, 128, 3, 2, 2, 1, 3, EPI_F32, 1>;
using CfgBf16x3n64 = TcCfg<KIND_BF16, 64, 4, 2, 2, 1, 3, EPI_F32, 1>;
// 256 x 128 tiles on CTA pairs, 4 stages of 48 KB per CTA.
using CfgBf16x3Pair = Tc2Cfg<KIND_BF16, 128, 4, 2, 2, 1, 3, EPI_F32, 1>;
// bf16 / f16 operands as given (one product): 128 x 128 single-CTA tiles with
// 6 stages of 32 KB, or 256 x 128 CTA-pair tiles with 8 stages of 24 KB per CTA.
using CfgHalf = TcCfg<KIND_BF16, 128, 6, 1, 1, 1, 1, EPI_F32, 1>;
using CfgHalfPair = Tc2Cfg<KIND_BF16, 128, 8, 1, 1, 1, 1, EPI_F32, 1>;
// 6 products (3 slices) on CTA pairs: 256 x 128 tiles, 3 stages of 72 KB per
// CTA, hi*hi and the corrections in two TMEM accumulators.
using CfgBf16x6Pair = Tc2Cfg<KIND_BF16, 128, 3, 3, 3, 2, 6, EPI_F32, 1>;
using CfgBf16x6 = TcCfg<KIND_BF16, 128, 2, 3, 3, 2, 6, EPI_F32, 1>;

// K blocks per TMEM accumulation chunk of the one-product bf16 / f16 GEMM
// (its MMAs are 3x shorter per K block than the split form's, so its chunks
// are longer to keep the epilogue's chunk sums off the critical path).
static int half_kchunk() {
    static int v = [] {
        const char* e = getenv("FG_HALF_KCHUNK");
        return e ? atoi(e) : 8;
    }();
    return v;
}

// K blocks (64 bf16 each) per TMEM accumulation chunk of the split SGEMM.
static int split_kchunk() {
    static int v = [] {
        const char* e = getenv("FG_SPLIT_KCHUNK");
        return e ? atoi(e) : 4;
    }();
    return v;
}

static unsigned long long kTimeoutNs = 4000000000ull;  // 4 s per wait

// Row tiles per raster group of the persistent tile walk: FG_RASTER when
// set, else 16 for the plain i8 CTA-pair kernel and 8 for the rest (B200,
// 8192^3, same box: i8 3.10-3.16 POPS at 16 against 3.00-3.05 at 8; the
// 3xBF16 pair kernel 479 TFLOP/s at 8 against 435-469 at 16, bf16 x bf16
// 1193 against 1130; the scheme II products and the quantized GEMM within
// noise of each other).
static int raster_env() {
    static int v = [] {
        const char* e = getenv("FG_RASTER");
        return e ? atoi(e) : 0;
    }();
    return v;
}
template <class Cfg>
static int raster_group() {
    if (raster_env() > 0) return raster_env();
    return (Cfg::KIND == KIND_I8 && Cfg::EPI == EPI_I32 && Cfg::BM == 256) ? 16 : 8;
}

template <class Cfg>
static const char* cfg_name() {
    if (Cfg::BM == 256)
        return Cfg::KIND == KIND_BF16
                   ? (Cfg::NOPS == 6 ? "tc_gemm2_6xbf16" : Cfg::NOPS == 3 ? "tc_gemm2_3xbf16" : "tc_gemm2_f16")
                   : "tc_gemm2_i8";
    if (Cfg::KIND == KIND_BF16)
        return Cfg::NOPS == 6 ? "tc_gemm_6xbf16" : Cfg::NOPS == 3 ? "tc_gemm_3xbf16" : "tc_gemm_f16";
    if (Cfg::EPI == EPI_I16) return "tc_gemm_i16";
    if (Cfg::EPI == EPI_QMM) return "tc_gemm_qmm";
    return "tc_gemm_i8";
}

static int grid_for_total(long long total) {
    return static_cast<int>(std::min<long long>(std::max<long long>((total + 255) / 256, 1), 4096));
}

template <class Cfg>
static fg_status launch_cfg(fg_ctx* ctx, const TcMaps& maps, TcArgs& args, cudaStream_t st) {
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(once, [] {
        attr_err = cudaFuncSetAttribute(tc_gemm_kernel<Cfg>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(tc_smem_bytes<Cfg>()));
    });
    FG_CUDA(attr_err);
    args.status = ctx->d_status;
    args.timeout_ns = kTimeoutNs;
    if (args.raster <= 0) args.raster = raster_group<Cfg>();
    const long long tiles =
        (long long)std::max(args.splits, 1) * args.batch * args.tiles_m * args.tiles_n;
    if (tiles == 0) return FG_OK;
    const int grid = static_cast<int>(std::min<long long>(tiles, ctx->sm_count));
    ProfScope prof(cfg_name<Cfg>(), st);
    tc_gemm_kernel<Cfg><<<grid, Cfg::THREADS, tc_smem_bytes<Cfg>(), st>>>(maps, args);
    prof.stop();
    count_launch();
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

// CTA-pair kernels: a persistent grid of as many pairs as can be resident
// (cudaOccupancyMaxActiveClusters; at most one pair per TPC).
template <class Cfg>
static fg_status launch_pair(fg_ctx* ctx, const TcMaps& maps, TcArgs& args, cudaStream_t st) {
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    static int max_pairs = 0;
    std::call_once(once, [ctx] {
        attr_err = cudaFuncSetAttribute(tc_gemm2_kernel<Cfg>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(tc2_smem_bytes<Cfg>()));
        if (attr_err != cudaSuccess) return;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(static_cast<unsigned>(ctx->sm_count & ~1), 1, 1);
        cfg.blockDim = dim3(Cfg::THREADS, 1, 1);
        cfg.dynamicSmemBytes = tc2_smem_bytes<Cfg>();
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, tc_gemm2_kernel<Cfg>, &cfg) == cudaSuccess && n > 0)
            max_pairs = n;
        else
            cudaGetLastError();
        if (max_pairs <= 0) max_pairs = ctx->sm_count / 2;
    });
    FG_CUDA(attr_err);
    args.status = ctx->d_status;
    args.timeout_ns = kTimeoutNs;
    if (args.raster <= 0) args.raster = raster_group<Cfg>();
    const long long units =
        (long long)std::max(args.splits, 1) * args.batch * args.tiles_m * args.tiles_n;
    if (units == 0) return FG_OK;
    const int grid = 2 * static_cast<int>(std::min<long long>(units, max_pairs));
    ProfScope prof(cfg_name<Cfg>(), st);
    tc_gemm2_kernel<Cfg><<<grid, Cfg::THREADS, tc2_smem_bytes<Cfg>(), st>>>(maps, args);
    prof.stop();
    count_launch();
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

template <class Cfg>
static fg_status launch_any(fg_ctx* ctx, const TcMaps& maps, TcArgs& args, cudaStream_t st) {
    if constexpr (Cfg::BM == 256)
        return launch_pair<Cfg>(ctx, maps, args, st);
    else
        return launch_cfg<Cfg>(ctx, maps, args, st);
}

// Launches Cfg with up to `want` K splits (tuned).  With more than one
// split the kernel writes dense partial products [split][batch][M][N] into a
// workspace and splitk_reduce_kernel combines them into C (wrapping int32
// sum + accumulate, or alpha * sum + beta * C).
template <class Cfg, typename T>
static fg_status launch_splitk(fg_ctx* ctx, const TcMaps& maps, TcArgs& args, int want, T* C,
                               long long ldc, long long strideC, T alpha, T beta, int accumulate,
                               cudaStream_t st) {
    const long long M = args.M, N = args.N, out_elems = M * N * args.batch;
    int kps = args.k_blocks;
    const int splits = plan_splits(want, args.k_blocks, out_elems, sizeof(T), &kps);
    if (splits <= 1) return launch_any<Cfg>(ctx, maps, args, st);
    Scratch ws;
    FG_TRY(ws.alloc(static_cast<size_t>(splits * out_elems) * sizeof(T), st));
    args.splits = splits;
    args.kb_per_split = kps;
    args.C = ws.p;
    args.ldc = N;
    args.strideC = M * N;
    args.accumulate = 0;
    args.alpha = 1.f;
    args.beta = 0.f;
    FG_TRY(launch_any<Cfg>(ctx, maps, args, st));
    splitk_reduce_kernel<T><<<grid_for_total(out_elems), 256, 0, st>>>(
        static_cast<const T*>(ws.p), splits, M, N, args.batch, C, ldc, strideC, alpha, beta,
        accumulate);
    count_launch();
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

// Operand map for a row-major matrix stack: inner = contiguous extent,
// rows = outer extent, `count` matrices `mstride_bytes` apart.
static fg_status operand_map(CUtensorMap* map, CUtensorMapDataType dt, const void* base,
                             long long inner, long long rows, long long ld_bytes, long long count,
                             long long mstride_bytes, uint32_t box_inner, uint32_t box_rows,
                             int* rank3) {
    uint64_t dims[3] = {static_cast<uint64_t>(inner), static_cast<uint64_t>(rows),
                        static_cast<uint64_t>(count)};
    uint64_t strides[2] = {static_cast<uint64_t>(ld_bytes), static_cast<uint64_t>(mstride_bytes)};
    uint32_t box[3] = {box_inner, box_rows, 1};
    *rank3 = count > 1 ? 1 : 0;
    return encode_map(map, dt, count > 1 ? 3 : 2, base, dims, strides, box);
}

static bool tma_ok(const void* p, long long ld_bytes, long long count, long long mstride_bytes) {
    if (reinterpret_cast<uintptr_t>(p) & 15) return false;
    if (ld_bytes % 16) return false;
    if (count > 1 && (mstride_bytes % 16)) return false;
    return true;
}

static long long round_up(long long x, long long a) { return (x + a - 1) / a * a; }

static void fill_batch(const Gemm& g, TcArgs& a) {
    a.batch = g.batch;
    a.bdims = g.bdims;
    for (int d = 0; d < 4; ++d) {
        a.bshape[d] = g.bshape[d];
        a.a_bstride[d] = g.a_istride[d];
        a.b_bstride[d] = g.b_istride[d];
    }
    a.strideC = g.c_stride;
}

static int grid_for(long long total) {
    return static_cast<int>(std::min<long long>(std::max<long long>((total + 255) / 256, 1), 4096));
}

// Copies an operand stack of 1-byte (or `esize`) rows into a 16-byte-pitched
// scratch buffer when its pointer/strides break the TMA rules.
static fg_status make_tma_operand(const void* src, long long rows, long long cols, long long ld,
                                  long long count, long long mstride, int esize, Scratch& sc,
                                  const void** out, long long* out_ld, long long* out_mstride,
                                  cudaStream_t st) {
    const long long ld_b = ld * esize, ms_b = mstride * esize;
    if (tma_ok(src, ld_b, count, ms_b)) {
        *out = src;
        *out_ld = ld;
        *out_mstride = mstride;
        return FG_OK;
    }
    const long long pitch = round_up(cols * esize, 16);
    FG_TRY(sc.alloc(static_cast<size_t>(pitch * rows * count), st));
    dim3 grid(grid_for(rows * cols * esize), static_cast<unsigned>(count));
    pad_rows_kernel<<<grid, 256, 0, st>>>(static_cast<const uint8_t*>(src), rows, cols * esize, ld_b,
                                          static_cast<uint8_t*>(sc.p), pitch, ms_b, pitch * rows);
    count_launch();
    FG_CUDA(cudaGetLastError());
    *out = sc.p;
    *out_ld = pitch / esize;
    *out_mstride = pitch * rows / esize;
    return FG_OK;
}

// Largest K one launch may cover with exact int32 accumulation.
static long long max_k_chunk(fg_dtype d) {
    switch (d) {
        case FG_I8: return 131072;   // |a*b| <= 2^14
        case FG_U8I8: return 65536;  // |a*b| <= 255*128
        case FG_I16: return 32768;   // byte-slice products <= 255^2 (two per mid term)
        default: return 1LL << 40;
    }
}

fg_status launch_int_tc(fg_ctx* ctx, const Gemm& g0, cudaStream_t st) {
    const long long kchunk = max_k_chunk(g0.dtype);
    if (g0.K > kchunk) {
        // Split K; later chunks accumulate into C (wrapping, so exact mod 2^32).
        for (long long k0 = 0; k0 < g0.K; k0 += kchunk) {
            Gemm g = g0;
            g.K = std::min(kchunk, g0.K - k0);
            g.A = static_cast<const uint8_t*>(g0.A) + k0 * in_size(g0.dtype);
            g.B = static_cast<const uint8_t*>(g0.B) + k0 * g0.ldb * in_size(g0.dtype);
            g.accumulate = (k0 == 0) ? g0.accumulate : 1;
            FG_TRY(launch_int_tc(ctx, g, st));
        }
        return FG_OK;
    }
    const Gemm& g = g0;
    TcMaps maps;
    TcArgs args{};
    args.M = static_cast<int>(g.M);
    args.N = static_cast<int>(g.N);
    args.K = static_cast<int>(g.K);
    args.tiles_m = static_cast<int>((g.M + 127) / 128);
    args.C = g.C;
    args.ldc = g.ldc;
    args.accumulate = g.accumulate;
    fill_batch(g, args);

    if (g.dtype == FG_I8 || g.dtype == FG_U8I8) {
        Scratch sa, sb;
        const void *pa, *pb;
        long long lda, ldb, msa, msb;
        FG_TRY(make_tma_operand(g.A, g.M, g.K, g.lda, g.a_count, g.a_mstride, 1, sa, &pa, &lda, &msa, st));
        FG_TRY(make_tma_operand(g.B, g.K, g.N, g.ldb, g.b_count, g.b_mstride, 1, sb, &pb, &ldb, &msb, st));
        FG_TRY(operand_map(&maps.a[0], CU_TENSOR_MAP_DATA_TYPE_UINT8, pa, g.K, g.M, lda, g.a_count, msa,
                           128, 128, &args.a_rank3));
        FG_TRY(operand_map(&maps.b[0], CU_TENSOR_MAP_DATA_TYPE_UINT8, pb, g.N, g.K, ldb, g.b_count, msb,
                           128, 128, &args.b_rank3));
        args.k_blocks = static_cast<int>((g.K + CfgI8::BK - 1) / CfgI8::BK);
        args.ops[0] = TcOp{0, 0, 0, g.dtype == FG_I8 ? 1 : 0, 1};
        const TuneChoice c = tune_lookup(TUNE_I8, g.M, g.N, g.K);
        int32_t* C = static_cast<int32_t*>(g.C);
        if (c.variant == 2) {
            args.tiles_m = static_cast<int>((g.M + CfgI8Pair::BM - 1) / CfgI8Pair::BM);
            args.tiles_n = static_cast<int>((g.N + CfgI8Pair::BN - 1) / CfgI8Pair::BN);
            return launch_splitk<CfgI8Pair, int32_t>(ctx, maps, args, c.splits, C, g.ldc, g.c_stride,
                                                     0, 0, g.accumulate, st);
        }
        if (c.variant == 3) {
            args.tiles_m = static_cast<int>((g.M + CfgI8PairW::BM - 1) / CfgI8PairW::BM);
            args.tiles_n = static_cast<int>((g.N + CfgI8PairW::TILE_N - 1) / CfgI8PairW::TILE_N);
            args.ops[1] = TcOp{0, 1, 1, g.dtype == FG_I8 ? 1 : 0, 1};
            return launch_splitk<CfgI8PairW, int32_t>(ctx, maps, args, c.splits, C, g.ldc, g.c_stride,
                                                      0, 0, g.accumulate, st);
        }
        if (c.variant == 1) {
            args.tiles_n = static_cast<int>((g.N + CfgI8n128::BN - 1) / CfgI8n128::BN);
            return launch_splitk<CfgI8n128, int32_t>(ctx, maps, args, c.splits, C, g.ldc, g.c_stride,
                                                     0, 0, g.accumulate, st);
        }
        args.tiles_n = static_cast<int>((g.N + CfgI8::BN - 1) / CfgI8::BN);
        return launch_splitk<CfgI8, int32_t>(ctx, maps, args, c.splits, C, g.ldc, g.c_stride, 0, 0,
                                             g.accumulate, st);
    }
    if (g.dtype == FG_I16) {
        // Byte slices, rows padded to 16 bytes.
        const long long pa = round_up(g.K, 16), pb = round_up(g.N, 16);
        const size_t a_bytes = static_cast<size_t>(pa * g.M * g.a_count);
        const size_t b_bytes = static_cast<size_t>(pb * g.K * g.b_count);
        Scratch s;
        FG_TRY(s.alloc(2 * a_bytes + 2 * b_bytes, st));
        int8_t* ahi = static_cast<int8_t*>(s.p);
        uint8_t* alo = reinterpret_cast<uint8_t*>(ahi + a_bytes);
        int8_t* bhi = reinterpret_cast<int8_t*>(alo + a_bytes);
        uint8_t* blo = reinterpret_cast<uint8_t*>(bhi + b_bytes);
        if (g.M * g.K > 0) {
            split_i16_kernel<<<dim3(grid_for(g.M * g.K), static_cast<unsigned>(g.a_count)), 256, 0, st>>>(
                static_cast<const int16_t*>(g.A), g.M, g.K, g.lda, ahi, alo, pa, g.a_mstride, pa * g.M);
            count_launch();
        }
        if (g.K * g.N > 0) {
            split_i16_kernel<<<dim3(grid_for(g.K * g.N), static_cast<unsigned>(g.b_count)), 256, 0, st>>>(
                static_cast<const int16_t*>(g.B), g.K, g.N, g.ldb, bhi, blo, pb, g.b_mstride, pb * g.K);
            count_launch();
        }
        FG_CUDA(cudaGetLastError());
        int r3;
        FG_TRY(operand_map(&maps.a[0], CU_TENSOR_MAP_DATA_TYPE_UINT8, ahi, g.K, g.M, pa, g.a_count, pa * g.M, 128, 128, &args.a_rank3));
        FG_TRY(operand_map(&maps.a[1], CU_TENSOR_MAP_DATA_TYPE_UINT8, alo, g.K, g.M, pa, g.a_count, pa * g.M, 128, 128, &r3));
        FG_TRY(operand_map(&maps.b[0], CU_TENSOR_MAP_DATA_TYPE_UINT8, bhi, g.N, g.K, pb, g.b_count, pb * g.K, 128, 128, &args.b_rank3));
        FG_TRY(operand_map(&maps.b[1], CU_TENSOR_MAP_DATA_TYPE_UINT8, blo, g.N, g.K, pb, g.b_count, pb * g.K, 128, 128, &r3));
        args.tiles_n = static_cast<int>((g.N + CfgI16::BN - 1) / CfgI16::BN);
        args.k_blocks = static_cast<int>((g.K + CfgI16::BK - 1) / CfgI16::BK);
        args.ops[0] = TcOp{0, 0, 0, 1, 1};  // hi*hi        -> acc0 (<<16)
        args.ops[1] = TcOp{0, 1, 1, 1, 0};  // hi(s8)*lo(u8) -> acc1 (<<8)
        args.ops[2] = TcOp{1, 0, 1, 0, 1};  // lo(u8)*hi(s8) -> acc1
        args.ops[3] = TcOp{1, 1, 2, 0, 0};  // lo*lo (u8)    -> acc2
        return launch_cfg<CfgI16>(ctx, maps, args, st);
    }
    return set_error(FG_ERR_DTYPE, "integer tensor-core path: unsupported dtype");
}

fg_status launch_qmm(fg_ctx* ctx, long long M, long long N, long long K, const uint8_t* a,
                     int a_zp, float scale, const int8_t* b, int b_zp, float* c, int accumulate,
                     cudaStream_t st) {
    if (K > max_k_chunk(FG_U8I8))
        return set_error(FG_ERR_UNSUPPORTED, "quantized_matmul: K above 65536 would overflow the exact i32 accumulator");
    Scratch sums;
    FG_TRY(sums.alloc(static_cast<size_t>((M + N) * sizeof(int)), st));
    int* row_sum = static_cast<int*>(sums.p);
    int* col_sum = row_sum + M;
    row_sum_u8_kernel<<<grid_for(M * 32), 256, 0, st>>>(a, M, K, K, row_sum);
    FG_CUDA(cudaMemsetAsync(col_sum, 0, N * sizeof(int), st));
    col_sum_i8_kernel<<<dim3(static_cast<unsigned>((N + 255) / 256), static_cast<unsigned>((K + 255) / 256)),
                        256, 0, st>>>(b, K, N, N, 256, col_sum);
    count_launch(2);
    FG_CUDA(cudaGetLastError());
    Scratch sa, sb;
    const void *pa, *pb;
    long long lda, ldb, msa, msb;
    FG_TRY(make_tma_operand(a, M, K, K, 1, 0, 1, sa, &pa, &lda, &msa, st));
    FG_TRY(make_tma_operand(b, K, N, N, 1, 0, 1, sb, &pb, &ldb, &msb, st));
    TcMaps maps;
    TcArgs args{};
    args.M = static_cast<int>(M);
    args.N = static_cast<int>(N);
    args.K = static_cast<int>(K);
    args.tiles_m = static_cast<int>((M + 127) / 128);
    args.tiles_n = static_cast<int>((N + CfgQmm::BN - 1) / CfgQmm::BN);
    args.k_blocks = static_cast<int>((K + CfgQmm::BK - 1) / CfgQmm::BK);
    args.batch = 1;
    args.C = c;
    args.ldc = N;
    args.accumulate = accumulate;
    args.row_sum = row_sum;
    args.col_sum = col_sum;
    args.a_zp = a_zp;
    args.b_zp = b_zp;
    args.scale = scale;
    args.ops[0] = TcOp{0, 0, 0, 0, 1};
    FG_TRY(operand_map(&maps.a[0], CU_TENSOR_MAP_DATA_TYPE_UINT8, pa, K, M, lda, 1, 0, 128, 128, &args.a_rank3));
    FG_TRY(operand_map(&maps.b[0], CU_TENSOR_MAP_DATA_TYPE_UINT8, pb, N, K, ldb, 1, 0, 128, 128, &args.b_rank3));
    // CTA pairs where the tuned i8 table picks them for this shape
    if (tune_lookup(TUNE_I8, M, N, K).variant == 2) {
        args.tiles_m = static_cast<int>((M + CfgQmmPair::BM - 1) / CfgQmmPair::BM);
        return launch_pair<CfgQmmPair>(ctx, maps, args, st);
    }
    return launch_cfg<CfgQmm>(ctx, maps, args, st);
}

// bf16 x bf16 / f16 x f16 -> f32 straight from the caller's 16-bit operands
// (gemm/mod.rs:851-933 widen them to f32 for an SGEMM): one tcgen05 kind::f16
// product per K block, K accumulated in TMEM chunks summed in FP32
// registers (round to nearest) like the split SGEMM; C = A@B, or C += A@B
// when accumulating.
fg_status launch_half_tc(fg_ctx* ctx, const Gemm& g, cudaStream_t st) {
    const CUtensorMapDataType tdt =
        g.dtype == FG_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
    const int fmt = g.dtype == FG_BF16 ? 1 : 0;  // kind::f16 operand format (0 F16, 1 BF16)
    Scratch sa, sb;
    const void *pa, *pb;
    long long lda, ldb, msa, msb;
    FG_TRY(make_tma_operand(g.A, g.M, g.K, g.lda, g.a_count, g.a_mstride, 2, sa, &pa, &lda, &msa, st));
    FG_TRY(make_tma_operand(g.B, g.K, g.N, g.ldb, g.b_count, g.b_mstride, 2, sb, &pb, &ldb, &msb, st));
    TcMaps maps;
    TcArgs args{};
    FG_TRY(operand_map(&maps.a[0], tdt, pa, g.K, g.M, lda * 2, g.a_count, msa * 2, 64, 128, &args.a_rank3));
    FG_TRY(operand_map(&maps.b[0], tdt, pb, g.N, g.K, ldb * 2, g.b_count, msb * 2, 64, 64, &args.b_rank3));
    args.M = static_cast<int>(g.M);
    args.N = static_cast<int>(g.N);
    args.K = static_cast<int>(g.K);
    args.tiles_m = static_cast<int>((g.M + 127) / 128);
    args.k_blocks = static_cast<int>((g.K + CfgHalf::BK - 1) / CfgHalf::BK);
    args.C = g.C;
    args.ldc = g.ldc;
    args.alpha = 1.f;
    args.beta = g.accumulate ? 1.f : 0.f;
    fill_batch(g, args);
    args.kchunk = half_kchunk();
    args.ops[0] = TcOp{0, 0, 0, fmt, fmt};
    float* C = static_cast<float*>(g.C);
    const TuneChoice c = tune_lookup(TUNE_SPLIT_F32, g.M, g.N, g.K);
    if (c.variant == 2) {
        args.tiles_m = static_cast<int>((g.M + CfgHalfPair::BM - 1) / CfgHalfPair::BM);
        args.tiles_n = static_cast<int>((g.N + CfgHalfPair::BN - 1) / CfgHalfPair::BN);
        return launch_splitk<CfgHalfPair, float>(ctx, maps, args, c.splits, C, g.ldc, g.c_stride, 1.f,
                                                 args.beta, 0, st);
    }
    args.tiles_n = static_cast<int>((g.N + CfgHalf::BN - 1) / CfgHalf::BN);
    return launch_splitk<CfgHalf, float>(ctx, maps, args, c.splits, C, g.ldc, g.c_stride, 1.f, args.beta, 0,
                                         st);
}

// 3xBF16: C = alpha * (Alo*Bhi + Ahi*Blo + Ahi*Bhi) + beta * C, f32 accumulate.
fg_status launch_split_bf16(fg_ctx* ctx, const Gemm& g, cudaStream_t st) {
    const bool cplx = g.dtype == FG_C32;
    if (cplx && g.batch > 1) {
        // Complex batches run one embedded product per output matrix.
        for (int i = 0; i < g.batch; ++i) {
            Gemm s = g;
            long long ia = 0, ib = 0;
            int rem = i;
            for (int d = g.bdims - 1; d >= 0; --d) {
                int idx = rem % g.bshape[d];
                rem /= g.bshape[d];
                ia += idx * g.a_istride[d];
                ib += idx * g.b_istride[d];
            }
            s.batch = 1;
            s.bdims = 0;
            s.a_count = s.b_count = 1;
            s.A = static_cast<const float2*>(g.A) + ia * g.a_mstride;
            s.B = static_cast<const float2*>(g.B) + ib * g.b_mstride;
            s.C = static_cast<float2*>(g.C) + i * g.c_stride;
            FG_TRY(launch_split_bf16(ctx, s, st));
        }
        return FG_OK;
    }
    // Real-embedded sizes for complex: (M x 2K) * (2K x 2N).
    const bool f16 = g.mode == FG_MODE_SPLIT_F16;  // two FP16 slices of scaled operands
    const int ns = (!f16 && g.slices == 3) ? 3 : 2;  // slices per operand
    const long long M = g.M, K = cplx ? 2 * g.K : g.K, N = cplx ? 2 * g.N : g.N;
    const long long pa = round_up(K, 8), pb = round_up(N, 8);  // bf16 elements, 16-byte pitch
    const size_t a_elems = static_cast<size_t>(pa * M * g.a_count);
    const size_t b_elems = static_cast<size_t>(pb * K * g.b_count);
    Scratch s;
    const size_t plane_bytes = (ns * a_elems + ns * b_elems) * sizeof(__nv_bfloat16);
    FG_TRY(s.alloc(round_up(plane_bytes, 256) + (f16 ? 256 : 0), st));
    BfPlanes ap{}, bp{};
    __nv_bfloat16* base = static_cast<__nv_bfloat16*>(s.p);
    for (int i = 0; i < ns; ++i) ap.p[i] = base + i * a_elems;
    for (int i = 0; i < ns; ++i) bp.p[i] = base + ns * a_elems + i * b_elems;
    unsigned* amax = nullptr;  // FP16 form: max |A| and max |B| as float bits
    if (f16) {
        amax = reinterpret_cast<unsigned*>(static_cast<uint8_t*>(s.p) + round_up(plane_bytes, 256));
        FG_CUDA(cudaMemsetAsync(amax, 0, 2 * sizeof(unsigned), st));
        // complex operands: max over the interleaved (re, im) floats
        const int cw = cplx ? 2 : 1;
        const unsigned ga = static_cast<unsigned>(std::max<long long>(1, std::min<long long>(
                                (g.M * g.K * cw * g.a_count / 4 + 255) / 256, 4LL * ctx->sm_count)));
        const unsigned gb = static_cast<unsigned>(std::max<long long>(1, std::min<long long>(
                                (g.K * g.N * cw * g.b_count / 4 + 255) / 256, 4LL * ctx->sm_count)));
        if (g.M * g.K > 0)
            amax_bits_kernel<<<ga, 256, 0, st>>>(static_cast<const float*>(g.A), g.M, g.K * cw, g.lda * cw,
                                                 g.a_count, g.a_mstride * cw, amax);
        if (g.K * g.N > 0)
            amax_bits_kernel<<<gb, 256, 0, st>>>(static_cast<const float*>(g.B), g.K, g.N * cw, g.ldb * cw,
                                                 g.b_count, g.b_mstride * cw, amax + 1);
        count_launch(2);
    }
    if (cplx && f16) {
        if (g.M * g.K > 0) {
            split_f16_cplx_a_kernel<<<grid_for(g.M * g.K), 256, 0, st>>>(static_cast<const float2*>(g.A), g.M,
                                                                         g.K, g.lda, ap, pa, amax);
            count_launch();
        }
        if (g.K * g.N > 0) {
            split_f16_cplx_b_kernel<<<grid_for(g.K * g.N), 256, 0, st>>>(static_cast<const float2*>(g.B), g.K,
                                                                         g.N, g.ldb, bp, pb, amax + 1);
            count_launch();
        }
    } else if (f16) {
        ProfScope prof("split_f16", st);
        if (M * K > 0) {
            const dim3 grid(static_cast<unsigned>(std::min<long long>(M, 8LL * ctx->sm_count)), static_cast<unsigned>(g.a_count));
            split_f16_kernel<<<grid, 256, 0, st>>>(static_cast<const float*>(g.A), M, K, g.lda, ap, pa, g.a_mstride,
                                                   pa * M, amax);
            count_launch();
        }
        if (K * N > 0) {
            const dim3 grid(static_cast<unsigned>(std::min<long long>(K, 8LL * ctx->sm_count)), static_cast<unsigned>(g.b_count));
            split_f16_kernel<<<grid, 256, 0, st>>>(static_cast<const float*>(g.B), K, N, g.ldb, bp, pb, g.b_mstride,
                                                   pb * K, amax + 1);
            count_launch();
        }
        prof.stop();
    } else if (cplx) {
        if (g.M * g.K > 0) {
            if (ns == 3)
                split_bf16_cplx_a_kernel<3><<<grid_for(g.M * g.K), 256, 0, st>>>(
                    static_cast<const float2*>(g.A), g.M, g.K, g.lda, ap, pa);
            else
                split_bf16_cplx_a_kernel<2><<<grid_for(g.M * g.K), 256, 0, st>>>(
                    static_cast<const float2*>(g.A), g.M, g.K, g.lda, ap, pa);
            count_launch();
        }
        if (g.K * g.N > 0) {
            if (ns == 3)
                split_bf16_cplx_b_kernel<3><<<grid_for(g.K * g.N), 256, 0, st>>>(
                    static_cast<const float2*>(g.B), g.K, g.N, g.ldb, bp, pb);
            else
                split_bf16_cplx_b_kernel<2><<<grid_for(g.K * g.N), 256, 0, st>>>(
                    static_cast<const float2*>(g.B), g.K, g.N, g.ldb, bp, pb);
            count_launch();
        }
    } else {
        ProfScope prof("split_bf16", st);
        if (M * K > 0) {
            const dim3 grid(static_cast<unsigned>(std::min<long long>(M, 8LL * ctx->sm_count)), static_cast<unsigned>(g.a_count));
            if (ns == 3)
                split_bf16_kernel_t<3><<<grid, 256, 0, st>>>(static_cast<const float*>(g.A), M, K, g.lda, ap, pa, g.a_mstride, pa * M);
            else
                split_bf16_kernel_t<2><<<grid, 256, 0, st>>>(static_cast<const float*>(g.A), M, K, g.lda, ap, pa, g.a_mstride, pa * M);
            count_launch();
        }
        if (K * N > 0) {
            const dim3 grid(static_cast<unsigned>(std::min<long long>(K, 8LL * ctx->sm_count)), static_cast<unsigned>(g.b_count));
            if (ns == 3)
                split_bf16_kernel_t<3><<<grid, 256, 0, st>>>(static_cast<const float*>(g.B), K, N, g.ldb, bp, pb, g.b_mstride, pb * K);
            else
                split_bf16_kernel_t<2><<<grid, 256, 0, st>>>(static_cast<const float*>(g.B), K, N, g.ldb, bp, pb, g.b_mstride, pb * K);
            count_launch();
        }
        prof.stop();
    }
    FG_CUDA(cudaGetLastError());
    TcMaps maps;
    TcArgs args{};
    int r3;
    const CUtensorMapDataType pdt = f16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
    for (int i = 0; i < ns; ++i) {
        FG_TRY(operand_map(&maps.a[i], pdt, ap.p[i], K, M, pa * 2, g.a_count, pa * M * 2, 64, 128, i == 0 ? &args.a_rank3 : &r3));
        FG_TRY(operand_map(&maps.b[i], pdt, bp.p[i], N, K, pb * 2, g.b_count, pb * K * 2, 64, 64, i == 0 ? &args.b_rank3 : &r3));
    }
    args.f16_amax = amax;
    args.M = static_cast<int>(M);
    args.N = static_cast<int>(N);
    args.K = static_cast<int>(K);
    args.tiles_m = static_cast<int>((M + 127) / 128);
    args.tiles_n = static_cast<int>((N + CfgBf16x3::BN - 1) / CfgBf16x3::BN);
    args.k_blocks = static_cast<int>((K + CfgBf16x3::BK - 1) / CfgBf16x3::BK);
    args.C = g.C;
    args.ldc = g.ldc;  // complex: in complex elements -> float pitch below
    args.alpha = static_cast<float>(g.alpha_re);
    args.beta = static_cast<float>(g.beta_re);
    fill_batch(g, args);
    if (cplx) {
        if (g.alpha_im != 0.0 || g.beta_im != 0.0)
            return set_error(FG_ERR_UNSUPPORTED, "split CGEMM: complex alpha/beta must be real");
        args.cplx_half = static_cast<int>(g.N);
        args.ldc = 2 * g.ldc;
    }
    args.kchunk = split_kchunk();
    if (ns == 3) {
        // hi*hi + (hi*mid + mid*hi) + (hi*lo + lo*hi + mid*mid), smallest first
        args.ops[0] = TcOp{2, 0, 1, 1, 1};
        args.ops[1] = TcOp{0, 2, 1, 1, 1};
        args.ops[2] = TcOp{1, 1, 1, 1, 1};
        args.ops[3] = TcOp{1, 0, 1, 1, 1};
        args.ops[4] = TcOp{0, 1, 1, 1, 1};
        args.ops[5] = TcOp{0, 0, 0, 1, 1};
        // the pair kernel where the tuned 3-product table picks a pair tile
        if (!cplx && tune_lookup(TUNE_SPLIT_F32, M, N, K).variant == 2) {
            args.tiles_m = static_cast<int>((M + CfgBf16x6Pair::BM - 1) / CfgBf16x6Pair::BM);
            args.tiles_n = static_cast<int>((N + CfgBf16x6Pair::BN - 1) / CfgBf16x6Pair::BN);
            return launch_pair<CfgBf16x6Pair>(ctx, maps, args, st);
        }
        return launch_cfg<CfgBf16x6>(ctx, maps, args, st);
    }
    const int sf = f16 ? 0 : 1;  // kind::f16 operand format: 0 F16, 1 BF16
    args.ops[0] = TcOp{1, 0, 0, sf, sf};  // lo * hi
    args.ops[1] = TcOp{0, 1, 0, sf, sf};  // hi * lo
    args.ops[2] = TcOp{0, 0, 0, sf, sf};  // hi * hi
    // Tuned tile variant / split-K (real products only; the complex
    // embedding's interleaving epilogue runs unsplit with 128-wide tiles).
    const TuneChoice c = cplx ? TuneChoice{0, 1} : tune_lookup(TUNE_SPLIT_F32, M, N, K);
    float* C = static_cast<float*>(g.C);
    const float alpha = args.alpha, beta = args.beta;
    if (c.variant == 2) {
        args.tiles_m = static_cast<int>((M + CfgBf16x3Pair::BM - 1) / CfgBf16x3Pair::BM);
        args.tiles_n = static_cast<int>((N + CfgBf16x3Pair::BN - 1) / CfgBf16x3Pair::BN);
        return launch_splitk<CfgBf16x3Pair, float>(ctx, maps, args, c.splits, C, g.ldc, g.c_stride,
                                                   alpha, beta, 0, st);
    }
    if (c.variant == 1) {
        args.tiles_n = static_cast<int>((N + CfgBf16x3n64::BN - 1) / CfgBf16x3n64::BN);
        return launch_splitk<CfgBf16x3n64, float>(ctx, maps, args, c.splits, C, g.ldc, g.c_stride,
                                                  alpha, beta, 0, st);
    }
    return launch_splitk<CfgBf16x3, float>(ctx, maps, args, c.splits, C, g.ldc, g.c_stride, alpha,
                                           beta, 0, st);
}

}  // namespace fgrt
