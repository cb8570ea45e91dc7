// gemm_simt.cu -- host launchers of the plain FP64 / FP32 / complex GEMMs
// (FP64 pipe and FFMA; see simt_gemm.cuh).
#include "prep_kernels.cuh"
#include "runtime.h"
#include "simt_gemm.cuh"
#include "dmma_gemm.cuh"
#include "ffma_sgemm.cuh"
#include "tune.h"

#include <algorithm>
#include <mutex>

namespace fgrt {

using namespace fg;

static BatchMap batch_map(const Gemm& g) {
    BatchMap bm{};
    bm.bdims = g.bdims;
    for (int d = 0; d < 4; ++d) {
        bm.bshape[d] = g.bshape[d];
        bm.a_bstride[d] = g.a_istride[d] * g.a_mstride;
        bm.b_bstride[d] = g.b_istride[d] * g.b_mstride;
    }
    bm.c_bstride = g.c_stride;
    return bm;
}

static int grid_for(long long total) {
    return static_cast<int>(std::min<long long>(std::max<long long>((total + 255) / 256, 1), 4096));
}

// Plain real GEMM with the tuned tile variant and split-K count.  Split-K
// writes `splits` partial products into a workspace and a combine pass
// applies alpha / beta (the partial sums are added in split order).
template <typename T, int TMM, int TNN>
static fg_status launch_simt_real(const Gemm& g, BatchMap bm, int splits_want, cudaStream_t st) {
    constexpr int BTM = 16 * TMM, BTN = 16 * TNN;
    constexpr long long KUNIT = 64;  // split granularity in K
    const long long kunits = (g.K + KUNIT - 1) / KUNIT;
    int kps = static_cast<int>(kunits);
    const int splits = plan_splits(splits_want, static_cast<int>(kunits), g.M * g.N * g.batch,
                                   sizeof(T), &kps);
    if ((long long)splits * g.batch > 65535) return set_error(FG_ERR_UNSUPPORTED, "batch above 65535");
    dim3 grid((g.N + BTN - 1) / BTN, (g.M + BTM - 1) / BTM, g.batch * splits);
    const T* A = static_cast<const T*>(g.A);
    const T* B = static_cast<const T*>(g.B);
    if (splits <= 1) {
        simt_gemm_real<T, 8, TMM, TNN><<<grid, 256, 0, st>>>((int)g.M, (int)g.N, (int)g.K, (T)g.alpha_re, A,
                                                       g.lda, B, g.ldb, (T)g.beta_re,
                                                       static_cast<T*>(g.C), g.ldc, bm, g.batch, (int)g.K);
        count_launch();
        FG_CUDA(cudaGetLastError());
        return FG_OK;
    }
    Scratch ws;
    const long long out_elems = g.M * g.N * g.batch;
    FG_TRY(ws.alloc(static_cast<size_t>(splits * out_elems) * sizeof(T), st));
    BatchMap wbm = bm;
    wbm.c_bstride = g.M * g.N;
    simt_gemm_real<T, 8, TMM, TNN><<<grid, 256, 0, st>>>((int)g.M, (int)g.N, (int)g.K, T(1), A, g.lda, B,
                                                   g.ldb, T(0), static_cast<T*>(ws.p), g.N, wbm,
                                                   g.batch, (int)(kps * KUNIT));
    splitk_reduce_kernel<T><<<grid_for(out_elems), 256, 0, st>>>(
        static_cast<const T*>(ws.p), splits, g.M, g.N, g.batch, static_cast<T*>(g.C), g.ldc,
        g.c_stride, (T)g.alpha_re, (T)g.beta_re, 0);
    count_launch(2);
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

// Plain DGEMM on the FP64 tensor path (DMMA), same split-K scheme.
template <class Cfg = DmmaCfg>
static fg_status launch_dmma(fg_ctx* ctx, const Gemm& g, BatchMap bm, int splits_want, cudaStream_t st) {
    (void)ctx;
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(once, [] {
        attr_err = cudaFuncSetAttribute(dmma_gemm_f64_kernel<Cfg>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(Cfg::SMEM));
    });
    FG_CUDA(attr_err);
    constexpr long long KUNIT = 64;
    const long long kunits = (g.K + KUNIT - 1) / KUNIT;
    int kps = static_cast<int>(kunits);
    const int splits = plan_splits(splits_want, static_cast<int>(kunits), g.M * g.N * g.batch,
                                   sizeof(double), &kps);
    if ((long long)splits * g.batch > 65535) return set_error(FG_ERR_UNSUPPORTED, "batch above 65535");
    dim3 grid((g.N + Cfg::BN - 1) / Cfg::BN, (g.M + Cfg::BM - 1) / Cfg::BM, g.batch * splits);
    const double* A = static_cast<const double*>(g.A);
    const double* B = static_cast<const double*>(g.B);
    if (splits <= 1) {
        dmma_gemm_f64_kernel<Cfg><<<grid, Cfg::THREADS, Cfg::SMEM, st>>>(
            (int)g.M, (int)g.N, (int)g.K, g.alpha_re, A, g.lda, B, g.ldb, g.beta_re,
            static_cast<double*>(g.C), g.ldc, bm, g.batch, (int)g.K);
        count_launch();
        FG_CUDA(cudaGetLastError());
        return FG_OK;
    }
    Scratch ws;
    const long long out_elems = g.M * g.N * g.batch;
    FG_TRY(ws.alloc(static_cast<size_t>(splits * out_elems) * sizeof(double), st));
    BatchMap wbm = bm;
    wbm.c_bstride = g.M * g.N;
    dmma_gemm_f64_kernel<Cfg><<<grid, Cfg::THREADS, Cfg::SMEM, st>>>(
        (int)g.M, (int)g.N, (int)g.K, 1.0, A, g.lda, B, g.ldb, 0.0, static_cast<double*>(ws.p), g.N, wbm,
        g.batch, (int)(kps * KUNIT));
    splitk_reduce_kernel<double><<<grid_for(out_elems), 256, 0, st>>>(
        static_cast<const double*>(ws.p), splits, g.M, g.N, g.batch, static_cast<double*>(g.C), g.ldc,
        g.c_stride, g.alpha_re, g.beta_re, 0);
    count_launch(2);
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

// Plain SGEMM on the cp.async FFMA kernel (ffma_sgemm.cuh): A transposed
// into packed scratch, B in place when aligned (else packed), same split-K
// scheme.  Results are bit-identical to simt_gemm_real<float, 8, 8, 8>.
template <class Cfg>
static fg_status launch_ffma(const Gemm& g, int splits_want, cudaStream_t st) {
    constexpr bool kSkinny = Cfg::BM == 32;
    auto kern = kSkinny ? ffma_sgemm_skinny_kernel : ffma_sgemm_kernel;
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(once, [kern] {
        attr_err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(Cfg::SMEM));
    });
    FG_CUDA(attr_err);
    const long long M = g.M, N = g.N, K = g.K;
    const long long Mp = (M + 3) / 4 * 4, Np = (N + 3) / 4 * 4;
    const float* A = static_cast<const float*>(g.A);
    const float* B = static_cast<const float*>(g.B);
    Scratch sa, sb;
    FG_TRY(sa.alloc(static_cast<size_t>(g.a_count * K * Mp) * sizeof(float), st));
    float* At = static_cast<float*>(sa.p);
    transpose_pack_kernel<<<dim3(static_cast<unsigned>((Mp + 31) / 32), static_cast<unsigned>((K + 31) / 32),
                                 static_cast<unsigned>(g.a_count)),
                            dim3(32, 8), 0, st>>>(A, (int)M, (int)K, g.lda, g.a_mstride, At, Mp);
    count_launch();
    const bool direct = (reinterpret_cast<uintptr_t>(B) % 16) == 0 && g.ldb % 4 == 0 && N % 4 == 0;
    const float* Bk = B;
    long long ldbk = g.ldb;
    BatchMap bm = batch_map(g);
    for (int d = 0; d < 4; ++d) bm.a_bstride[d] = g.a_istride[d] * K * Mp;
    if (!direct) {
        FG_TRY(sb.alloc(static_cast<size_t>(g.b_count * K * Np) * sizeof(float), st));
        float* Bp = static_cast<float*>(sb.p);
        pack_rows_kernel<<<dim3(static_cast<unsigned>(std::min<long long>((K * Np + 255) / 256, 4096)),
                                static_cast<unsigned>(g.b_count)),
                           256, 0, st>>>(B, (int)K, (int)N, g.ldb, g.b_mstride, Bp, Np);
        count_launch();
        Bk = Bp;
        ldbk = Np;
        for (int d = 0; d < 4; ++d) bm.b_bstride[d] = g.b_istride[d] * K * Np;
    }
    const int bcols = static_cast<int>(direct ? N : Np);
    constexpr long long KUNIT = 64;
    const long long kunits = (K + KUNIT - 1) / KUNIT;
    int kps = static_cast<int>(kunits);
    const int splits = plan_splits(splits_want, static_cast<int>(kunits), M * N * g.batch, sizeof(float), &kps);
    if ((long long)splits * g.batch > 65535) return set_error(FG_ERR_UNSUPPORTED, "batch above 65535");
    dim3 grid((N + Cfg::BN - 1) / Cfg::BN, (M + Cfg::BM - 1) / Cfg::BM, g.batch * splits);
    if (splits <= 1) {
        kern<<<grid, Cfg::THREADS, Cfg::SMEM, st>>>(
            (int)M, (int)N, (int)K, (float)g.alpha_re, At, Mp, Bk, ldbk, bcols, (float)g.beta_re,
            static_cast<float*>(g.C), g.ldc, bm, g.batch, (int)K);
        count_launch();
        FG_CUDA(cudaGetLastError());
        return FG_OK;
    }
    Scratch ws;
    const long long out_elems = M * N * g.batch;
    FG_TRY(ws.alloc(static_cast<size_t>(splits * out_elems) * sizeof(float), st));
    BatchMap wbm = bm;
    wbm.c_bstride = M * N;
    kern<<<grid, Cfg::THREADS, Cfg::SMEM, st>>>(
        (int)M, (int)N, (int)K, 1.f, At, Mp, Bk, ldbk, bcols, 0.f, static_cast<float*>(ws.p), N, wbm, g.batch,
        (int)(kps * KUNIT));
    splitk_reduce_kernel<float><<<grid_for(out_elems), 256, 0, st>>>(
        static_cast<const float*>(ws.p), splits, M, N, g.batch, static_cast<float*>(g.C), g.ldc, g.c_stride,
        (float)g.alpha_re, (float)g.beta_re, 0);
    count_launch(2);
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

// Matrix-vector shapes (one operand is a vector; ferray's matmul of a 1-D
// operand, products/mod.rs:362-437) go to the GEMV kernels.
template <typename T>
static fg_status launch_gemv(fg_ctx* ctx, const Gemm& g, cudaStream_t st) {
    const T* A = static_cast<const T*>(g.A);
    const T* B = static_cast<const T*>(g.B);
    T* C = static_cast<T*>(g.C);
    if (g.N == 1) {
        const long long blocks = (g.M * 32 + 255) / 256;
        gemv_rows_kernel<T><<<static_cast<unsigned>(blocks), 256, 0, st>>>(
            (int)g.M, (int)g.K, (T)g.alpha_re, A, g.lda, B, g.ldb, (T)g.beta_re, C, g.ldc);
        count_launch();
        FG_CUDA(cudaGetLastError());
        return FG_OK;
    }
    constexpr int CW = 32 * (16 / sizeof(T));
    const long long cblocks = (g.N + CW - 1) / CW;
    // split K across blocks until there are about 4 blocks per SM
    int splits = static_cast<int>(std::min<long long>(
        std::max<long long>(1, (4LL * ctx->sm_count) / cblocks), std::max<long long>(1, g.K / 256)));
    splits = std::min(splits, 64);
    const int ksplit = static_cast<int>((g.K + splits - 1) / splits);
    splits = static_cast<int>((g.K + ksplit - 1) / ksplit);
    dim3 grid(static_cast<unsigned>(cblocks), static_cast<unsigned>(splits));
    if (splits == 1) {
        gemv_cols_kernel<T><<<grid, 256, 0, st>>>((int)g.N, (int)g.K, ksplit, (T)g.alpha_re, A, 1, B,
                                                  g.ldb, (T)g.beta_re, C, 0);
        count_launch();
        FG_CUDA(cudaGetLastError());
        return FG_OK;
    }
    Scratch ws;
    FG_TRY(ws.alloc(static_cast<size_t>(splits * g.N) * sizeof(T), st));
    gemv_cols_kernel<T><<<grid, 256, 0, st>>>((int)g.N, (int)g.K, ksplit, (T)g.alpha_re, A, 1, B, g.ldb,
                                              (T)g.beta_re, static_cast<T*>(ws.p), g.N);
    splitk_reduce_kernel<T><<<grid_for(g.N), 256, 0, st>>>(static_cast<const T*>(ws.p), splits, 1, g.N, 1,
                                                           C, g.ldc, 0, (T)g.alpha_re, (T)g.beta_re, 0);
    count_launch(2);
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

fg_status launch_simt(fg_ctx* ctx, const Gemm& g, cudaStream_t st) {
    if (g.batch == 1 && (g.N == 1 || g.M == 1) && (g.dtype == FG_F64 || g.dtype == FG_F32)) {
        ProfScope prof(g.dtype == FG_F64 ? "gemv_f64" : "gemv_f32", st);
        return g.dtype == FG_F64 ? launch_gemv<double>(ctx, g, st) : launch_gemv<float>(ctx, g, st);
    }
    const BatchMap bm = batch_map(g);
    if (g.batch > 65535) return set_error(FG_ERR_UNSUPPORTED, "batch above 65535");
    static const char* names[] = {"simt_dgemm", "simt_sgemm", "simt_zgemm", "simt_cgemm"};
    const char* fam = g.dtype <= FG_C32 ? names[g.dtype] : "simt";
    if (g.dtype == FG_F64 || g.dtype == FG_F32) {  // profile under the tuned kernel's name
        const TuneChoice c = tune_lookup(g.dtype == FG_F64 ? TUNE_F64 : TUNE_F32, g.M, g.N, g.K);
        if (c.variant == 4) fam = g.dtype == FG_F64 ? "dmma_dgemm" : "ffma_sgemm";
        if (c.variant == 5) fam = g.dtype == FG_F64 ? "dmma_dgemm_skinny" : "ffma_sgemm_skinny";
    }
    ProfScope prof(fam, st);
    switch (g.dtype) {
        case FG_F64: {
            const TuneChoice c = tune_lookup(TUNE_F64, g.M, g.N, g.K);
            switch (c.variant) {
                case 1: return launch_simt_real<double, 4, 4>(g, bm, c.splits, st);
                case 2: return launch_simt_real<double, 2, 8>(g, bm, c.splits, st);
                case 3: return launch_simt_real<double, 8, 2>(g, bm, c.splits, st);
                case 4: return launch_dmma(ctx, g, bm, c.splits, st);
                case 5: return launch_dmma<DmmaSkinnyCfg>(ctx, g, bm, c.splits, st);
                default: return launch_simt_real<double, 8, 8>(g, bm, c.splits, st);
            }
        }
        case FG_F32: {
            const TuneChoice c = tune_lookup(TUNE_F32, g.M, g.N, g.K);
            switch (c.variant) {
                case 1: return launch_simt_real<float, 4, 4>(g, bm, c.splits, st);
                case 2: return launch_simt_real<float, 2, 8>(g, bm, c.splits, st);
                case 3: return launch_simt_real<float, 8, 2>(g, bm, c.splits, st);
                case 4:
                    // the packed transpose wants a K grid below 65536 blocks
                    if (g.M > 0 && g.N > 0 && g.K > 0 && g.K <= 32LL * 65535)
                        return launch_ffma<FfmaCfg>(g, c.splits, st);
                    return launch_simt_real<float, 8, 8>(g, bm, c.splits, st);
                case 5:
                    if (g.M > 0 && g.N > 0 && g.K > 0 && g.K <= 32LL * 65535)
                        return launch_ffma<FfmaSkinnyCfg>(g, c.splits, st);
                    return launch_simt_real<float, 2, 8>(g, bm, c.splits, st);
                default: return launch_simt_real<float, 8, 8>(g, bm, c.splits, st);
            }
        }
        case FG_C64: {
            // Real scalars and one output matrix: the real-embedded GEMM on
            // the DMMA kernel (same 8MNK flops, FP64 FMA per product).
            if (g.batch == 1 && g.alpha_im == 0.0 && g.beta_im == 0.0 && g.K > 0 &&
                (reinterpret_cast<uintptr_t>(g.B) & 15) == 0) {  // 16-byte complex loads of B
                Scratch bx;
                FG_TRY(bx.alloc(static_cast<size_t>(4 * g.K * g.N) * sizeof(double), st));
                zgemm_expand_b_kernel<<<grid_for(g.K * g.N), 256, 0, st>>>(
                    static_cast<const double2*>(g.B), g.K, g.N, g.ldb, static_cast<double*>(bx.p));
                count_launch();
                Gemm r = g;
                r.dtype = FG_F64;
                r.M = g.M;
                r.N = 2 * g.N;
                r.K = 2 * g.K;
                r.lda = 2 * g.lda;
                r.B = bx.p;
                r.ldb = 2 * g.N;
                r.ldc = 2 * g.ldc;
                const TuneChoice c = tune_lookup(TUNE_F64, r.M, r.N, r.K);
                return launch_dmma(ctx, r, batch_map(r), c.variant == 4 ? c.splits : 1, st);
            }
            dim3 grid((g.N + 63) / 64, (g.M + 63) / 64, g.batch);
            simt_gemm_cplx<double, 8><<<grid, 256, 0, st>>>(
                (int)g.M, (int)g.N, (int)g.K, g.alpha_re, g.alpha_im,
                static_cast<const Cplx<double>*>(g.A), g.lda, static_cast<const Cplx<double>*>(g.B),
                g.ldb, g.beta_re, g.beta_im, static_cast<Cplx<double>*>(g.C), g.ldc, bm);
            break;
        }
        case FG_C32: {
            // Real scalars, one output matrix and a tuned f32 choice of the
            // cp.async FFMA kernel for the embedded shape: the real-embedded
            // GEMM (M x 2K) (2K x 2N) on it (same 8MNK flops, one FMA per
            // product); otherwise the 4M kernel.
            if (g.batch == 1 && g.alpha_im == 0.0 && g.beta_im == 0.0 && g.M > 0 && g.N > 0 && g.K > 0 &&
                2 * g.K <= 32LL * 65535 && (reinterpret_cast<uintptr_t>(g.B) & 7) == 0) {
                const TuneChoice c = tune_lookup(TUNE_F32, g.M, 2 * g.N, 2 * g.K);
                if (c.variant == 4) {
                    Scratch bx;
                    FG_TRY(bx.alloc(static_cast<size_t>(4 * g.K * g.N) * sizeof(float), st));
                    cgemm_expand_b_kernel<<<grid_for(g.K * g.N), 256, 0, st>>>(
                        static_cast<const float2*>(g.B), g.K, g.N, g.ldb, static_cast<float*>(bx.p));
                    count_launch();
                    Gemm r = g;
                    r.dtype = FG_F32;
                    r.N = 2 * g.N;
                    r.K = 2 * g.K;
                    r.lda = 2 * g.lda;
                    r.B = bx.p;
                    r.ldb = 2 * g.N;
                    r.ldc = 2 * g.ldc;
                    return launch_ffma<FfmaCfg>(r, c.splits, st);
                }
            }
            dim3 grid((g.N + 63) / 64, (g.M + 63) / 64, g.batch);
            simt_gemm_cplx<float, 8><<<grid, 256, 0, st>>>(
                (int)g.M, (int)g.N, (int)g.K, (float)g.alpha_re, (float)g.alpha_im,
                static_cast<const Cplx<float>*>(g.A), g.lda, static_cast<const Cplx<float>*>(g.B),
                g.ldb, (float)g.beta_re, (float)g.beta_im, static_cast<Cplx<float>*>(g.C), g.ldc, bm);
            break;
        }
        default:
            return set_error(FG_ERR_DTYPE, "SIMT path handles f64/f32/c64/c32 only");
    }
    count_launch();
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

}  // namespace fgrt
