// gemm_simt.cu -- host launchers of the plain FP64 / FP32 / complex GEMMs
// (FP64 pipe and FFMA; see simt_gemm.cuh).
#include "prep_kernels.cuh"
#include "runtime.h"
#include "simt_gemm.cuh"

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

fg_status launch_simt(fg_ctx* ctx, const Gemm& g, cudaStream_t st) {
    (void)ctx;
    const BatchMap bm = batch_map(g);
    if (g.batch > 65535) return set_error(FG_ERR_UNSUPPORTED, "batch above 65535");
    static const char* names[] = {"simt_dgemm", "simt_sgemm", "simt_zgemm", "simt_cgemm"};
    ProfScope prof(g.dtype <= FG_C32 ? names[g.dtype] : "simt", st);
    switch (g.dtype) {
        case FG_F64: {
            dim3 grid((g.N + 127) / 128, (g.M + 127) / 128, g.batch);
            simt_gemm_real<double, 8><<<grid, 256, 0, st>>>(
                (int)g.M, (int)g.N, (int)g.K, g.alpha_re, static_cast<const double*>(g.A), g.lda,
                static_cast<const double*>(g.B), g.ldb, g.beta_re, static_cast<double*>(g.C), g.ldc, bm);
            break;
        }
        case FG_F32: {
            dim3 grid((g.N + 127) / 128, (g.M + 127) / 128, g.batch);
            simt_gemm_real<float, 8><<<grid, 256, 0, st>>>(
                (int)g.M, (int)g.N, (int)g.K, (float)g.alpha_re, static_cast<const float*>(g.A), g.lda,
                static_cast<const float*>(g.B), g.ldb, (float)g.beta_re, static_cast<float*>(g.C), g.ldc, bm);
            break;
        }
        case FG_C64: {
            dim3 grid((g.N + 63) / 64, (g.M + 63) / 64, g.batch);
            simt_gemm_cplx<double, 8><<<grid, 256, 0, st>>>(
                (int)g.M, (int)g.N, (int)g.K, g.alpha_re, g.alpha_im,
                static_cast<const Cplx<double>*>(g.A), g.lda, static_cast<const Cplx<double>*>(g.B),
                g.ldb, g.beta_re, g.beta_im, static_cast<Cplx<double>*>(g.C), g.ldc, bm);
            break;
        }
        case FG_C32: {
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
