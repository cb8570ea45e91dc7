// api.cu -- the C ABI (include/ferray_gpu.h): context, buffers, argument
// lowering of every GEMM entry point to one internal Gemm description, the
// NumPy matmul shape logic, and dispatch to the kernel families.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "prep_kernels.cuh"
#include "runtime.h"

namespace fgrt {

using fg::scale_kernel;

std::atomic<uint64_t> g_launches{0};
std::atomic<int> g_prof_on{0};

struct ProfRec {
    std::string fam;
    cudaEvent_t e0, e1;
};
static std::mutex g_prof_mu;
static std::vector<ProfRec> g_prof;

void prof_record(const char* family, cudaEvent_t start, cudaEvent_t stop) {
    std::lock_guard<std::mutex> lk(g_prof_mu);
    g_prof.push_back(ProfRec{family, start, stop});
}
static thread_local std::string t_last_error;

fg_status set_error(fg_status s, const std::string& msg) {
    t_last_error = msg;
    return s;
}

fg_status cuda_error(cudaError_t e, const char* what) {
    t_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation) return FG_ERR_OOM;
    return FG_ERR_DEVICE;
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

fg_status encode_map(CUtensorMap* map, CUtensorMapDataType dt, int rank, const void* base,
                     const uint64_t* dims, const uint64_t* strides_bytes, const uint32_t* box) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return set_error(FG_ERR_DEVICE, "cuTensorMapEncodeTiled unavailable");
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = fn(map, dt, static_cast<cuuint32_t>(rank), const_cast<void*>(base),
                    reinterpret_cast<const cuuint64_t*>(dims),
                    reinterpret_cast<const cuuint64_t*>(strides_bytes),
                    reinterpret_cast<const cuuint32_t*>(box), estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return set_error(FG_ERR_INVALID, "cuTensorMapEncodeTiled failed (code " + std::to_string((int)r) + ")");
    return FG_OK;
}

static int grid_for(long long total) {
    return static_cast<int>(std::min<long long>(std::max<long long>((total + 255) / 256, 1), 4096));
}

// K == 0: C = beta*C (floats) or C = 0 / unchanged (integers), per batch.
// One thread waits, with the kernels' bounded wait, on an mbarrier that
// nothing ever arrives on: the wait gives up after timeout_ns, records
// FG_DEV_ERR_TIMEOUT at site 0x7F in the context's status word and the
// kernel returns normally (no fault, the context stays usable).
static __global__ void wait_probe_kernel(fg::DevStatus* st, uint64_t timeout_ns) {
    __shared__ uint64_t bar;
    __shared__ int abort_flag;
    if (threadIdx.x == 0) {
        fg::mbar_init(&bar, 1);
        abort_flag = 0;
        fg::fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) fg::mbar_wait(&bar, 0, timeout_ns, st, 0x7F, &abort_flag);
    __syncthreads();
}

static fg_status k_zero(const Gemm& g, cudaStream_t st) {
    for (int i = 0; i < g.batch; ++i) {
        switch (g.dtype) {
            case FG_F64:
                scale_kernel<double><<<grid_for(g.M * g.N), 256, 0, st>>>(
                    static_cast<double*>(g.C) + i * g.c_stride, g.M, g.N, g.ldc, g.beta_re);
                break;
            case FG_F32:
                scale_kernel<float><<<grid_for(g.M * g.N), 256, 0, st>>>(
                    static_cast<float*>(g.C) + i * g.c_stride, g.M, g.N, g.ldc, (float)g.beta_re);
                break;
            case FG_C64:
            case FG_C32:
                if (g.beta_im != 0.0)
                    return set_error(FG_ERR_UNSUPPORTED, "k == 0 with complex beta");
                if (g.dtype == FG_C64)
                    scale_kernel<double><<<grid_for(g.M * g.N * 2), 256, 0, st>>>(
                        static_cast<double*>(g.C) + 2 * i * g.c_stride, g.M, 2 * g.N, 2 * g.ldc, g.beta_re);
                else
                    scale_kernel<float><<<grid_for(g.M * g.N * 2), 256, 0, st>>>(
                        static_cast<float*>(g.C) + 2 * i * g.c_stride, g.M, 2 * g.N, 2 * g.ldc, (float)g.beta_re);
                break;
            default:
                if (g.accumulate) return FG_OK;
                scale_kernel<int><<<grid_for(g.M * g.N), 256, 0, st>>>(
                    static_cast<int*>(g.C) + i * g.c_stride, g.M, g.N, g.ldc, 0);
        }
        count_launch();
    }
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

fg_status run_gemm(fg_ctx* ctx, const Gemm& g, cudaStream_t st) {
    if (g.M < 0 || g.N < 0 || g.K < 0) return set_error(FG_ERR_SHAPE, "negative dimension");
    if (g.M == 0 || g.N == 0 || g.batch == 0) return FG_OK;
    if (!g.C || (g.K > 0 && (!g.A || !g.B))) return set_error(FG_ERR_INVALID, "null operand pointer");
    if (g.M > INT32_MAX / 2 || g.N > INT32_MAX / 2 || g.K > INT32_MAX / 2)
        return set_error(FG_ERR_UNSUPPORTED, "dimension above 2^30");
    if (g.lda < g.K || g.ldb < g.N || g.ldc < g.N)
        return set_error(FG_ERR_SHAPE, "leading dimension smaller than the row length");
    if (g.K == 0) return k_zero(g, st);
    switch (g.dtype) {
        case FG_F64:
        case FG_C64:
            return g.mode != FG_MODE_PLAIN ? launch_ozaki(ctx, g, st) : launch_simt(ctx, g, st);
        case FG_F32:
        case FG_C32:
            return g.mode != FG_MODE_PLAIN ? launch_split_bf16(ctx, g, st) : launch_simt(ctx, g, st);
        case FG_I8:
        case FG_U8I8:
        case FG_I16:
            return launch_int_tc(ctx, g, st);
        case FG_BF16:
        case FG_F16:
            return launch_half_tc(ctx, g, st);
    }
    return set_error(FG_ERR_DTYPE, "unknown dtype");
}

static bool valid_dtype(fg_dtype d) { return d >= FG_F64 && d <= FG_F16; }

static void set_scalars(Gemm& g, const void* alpha, const void* beta) {
    switch (g.dtype) {
        case FG_F64:
            g.alpha_re = alpha ? *static_cast<const double*>(alpha) : 1.0;
            g.beta_re = beta ? *static_cast<const double*>(beta) : 0.0;
            break;
        case FG_F32:
            g.alpha_re = alpha ? *static_cast<const float*>(alpha) : 1.0;
            g.beta_re = beta ? *static_cast<const float*>(beta) : 0.0;
            break;
        case FG_C64:
            if (alpha) { g.alpha_re = static_cast<const double*>(alpha)[0]; g.alpha_im = static_cast<const double*>(alpha)[1]; }
            if (beta) { g.beta_re = static_cast<const double*>(beta)[0]; g.beta_im = static_cast<const double*>(beta)[1]; }
            break;
        case FG_C32:
            if (alpha) { g.alpha_re = static_cast<const float*>(alpha)[0]; g.alpha_im = static_cast<const float*>(alpha)[1]; }
            if (beta) { g.beta_re = static_cast<const float*>(beta)[0]; g.beta_im = static_cast<const float*>(beta)[1]; }
            break;
        default:
            break;
    }
}

}  // namespace fgrt

using namespace fgrt;

extern "C" {

const char* fg_status_string(fg_status s) {
    switch (s) {
        case FG_OK: return "ok";
        case FG_ERR_SHAPE: return "shape mismatch";
        case FG_ERR_DTYPE: return "invalid dtype";
        case FG_ERR_OOM: return "device out of memory";
        case FG_ERR_BUDGET: return "HBM budget exceeded";
        case FG_ERR_TIMEOUT: return "timeout";
        case FG_ERR_DEVICE: return "CUDA error";
        case FG_ERR_INVALID: return "invalid argument";
        case FG_ERR_UNSUPPORTED: return "unsupported";
        case FG_ERR_BROADCAST: return "broadcast failure";
    }
    return "unknown";
}

const char* fg_last_error(void) { return t_last_error.c_str(); }

uint64_t fg_launch_count(void) { return g_launches.load(); }

fg_status fg_profile_enable(int on) {
    g_prof_on.store(on ? 1 : 0);
    return FG_OK;
}

fg_status fg_profile_collect(fg_profile_entry* out, int capacity, int* count) {
    std::vector<ProfRec> recs;
    {
        std::lock_guard<std::mutex> lk(g_prof_mu);
        recs.swap(g_prof);
    }
    std::vector<fg_profile_entry> agg;
    fg_status st = FG_OK;
    for (auto& r : recs) {
        float ms = 0.f;
        if (cudaEventSynchronize(r.e1) != cudaSuccess || cudaEventElapsedTime(&ms, r.e0, r.e1) != cudaSuccess)
            st = set_error(FG_ERR_DEVICE, "profile event failed");
        cudaEventDestroy(r.e0);
        cudaEventDestroy(r.e1);
        fg_profile_entry* e = nullptr;
        for (auto& x : agg)
            if (r.fam == x.name) e = &x;
        if (!e) {
            agg.push_back(fg_profile_entry{});
            e = &agg.back();
            std::strncpy(e->name, r.fam.c_str(), sizeof(e->name) - 1);
        }
        e->launches += 1;
        e->total_ms += ms;
    }
    int n = 0;
    for (auto& x : agg) {
        if (out && n < capacity) out[n] = x;
        ++n;
    }
    if (count) *count = n;
    return st;
}

fg_status fg_init(int device, fg_ctx** out) {
    if (!out) return set_error(FG_ERR_INVALID, "out is null");
    *out = nullptr;
    int n = 0;
    FG_CUDA(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) return set_error(FG_ERR_INVALID, "no such device");
    cudaDeviceProp prop;
    FG_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10)
        return set_error(FG_ERR_UNSUPPORTED, "this backend is built for sm_100 (B200); found sm_" +
                                                  std::to_string(prop.major * 10 + prop.minor));
    FG_CUDA(cudaSetDevice(device));
    fg_ctx* ctx = new fg_ctx();
    ctx->device = device;
    ctx->sm_count = prop.multiProcessorCount;
    ctx->cc_major = prop.major;
    ctx->cc_minor = prop.minor;
    ctx->hbm_bytes = prop.totalGlobalMem;
    cudaError_t e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->pipe_comp, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->pipe_out, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&ctx->d_status, sizeof(fg::DevStatus));
    if (e == cudaSuccess) e = cudaMemset(ctx->d_status, 0, sizeof(fg::DevStatus));
    if (e != cudaSuccess) {
        delete ctx;
        return cuda_error(e, "fg_init");
    }
    // Keep freed scratch cached in the stream-ordered pool between calls.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    *out = ctx;
    return FG_OK;
}

fg_status fg_shutdown(fg_ctx* ctx) {
    if (!ctx) return FG_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->pipe_comp) cudaStreamSynchronize(ctx->pipe_comp);
    if (ctx->pipe_out) cudaStreamSynchronize(ctx->pipe_out);
    cudaFree(ctx->d_status);
    if (ctx->pipe_comp) cudaStreamDestroy(ctx->pipe_comp);
    if (ctx->pipe_out) cudaStreamDestroy(ctx->pipe_out);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return FG_OK;
}

fg_status fg_sync(fg_ctx* ctx, fg_stream stream) {
    if (!ctx) return set_error(FG_ERR_INVALID, "null context");
    FG_CUDA(cudaSetDevice(ctx->device));
    FG_CUDA(cudaStreamSynchronize(stream_of(ctx, stream)));
    fg::DevStatus h{};
    FG_CUDA(cudaMemcpy(&h, ctx->d_status, sizeof(h), cudaMemcpyDeviceToHost));
    if (h.code != FG_DEV_OK) {
        FG_CUDA(cudaMemset(ctx->d_status, 0, sizeof(fg::DevStatus)));
        return set_error(h.code == FG_DEV_ERR_TIMEOUT ? FG_ERR_TIMEOUT : FG_ERR_DEVICE,
                         "kernel reported error " + std::to_string(h.code) + " at site " +
                             std::to_string(h.where) + " (block " + std::to_string(h.block) + ")");
    }
    return FG_OK;
}

fg_status fg_selftest_wait_timeout(fg_ctx* ctx, uint32_t timeout_us, fg_stream stream) {
    if (!ctx) return set_error(FG_ERR_INVALID, "null context");
    if (timeout_us == 0 || timeout_us > 1000000)
        return set_error(FG_ERR_INVALID, "fg_selftest_wait_timeout: timeout outside 1 us .. 1 s");
    FG_CUDA(cudaSetDevice(ctx->device));
    wait_probe_kernel<<<1, 32, 0, stream_of(ctx, stream)>>>(ctx->d_status, 1000ull * timeout_us);
    count_launch();
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

fg_status fg_device_info(fg_ctx* ctx, int* sm_count, int* cc_major, int* cc_minor,
                         size_t* hbm_bytes) {
    if (!ctx) return set_error(FG_ERR_INVALID, "null context");
    if (sm_count) *sm_count = ctx->sm_count;
    if (cc_major) *cc_major = ctx->cc_major;
    if (cc_minor) *cc_minor = ctx->cc_minor;
    if (hbm_bytes) *hbm_bytes = ctx->hbm_bytes;
    return FG_OK;
}

fg_status fg_buffer_alloc(fg_ctx* ctx, size_t bytes, void** dptr) {
    if (!ctx || !dptr) return set_error(FG_ERR_INVALID, "null argument");
    FG_CUDA(cudaSetDevice(ctx->device));
    cudaError_t e = cudaMalloc(dptr, bytes ? bytes : 16);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *dptr = nullptr;
        return set_error(FG_ERR_OOM, "device allocation of " + std::to_string(bytes) + " bytes failed");
    }
    return FG_OK;
}

fg_status fg_buffer_free(fg_ctx* ctx, void* dptr) {
    if (!ctx) return set_error(FG_ERR_INVALID, "null context");
    if (!dptr) return FG_OK;
    FG_CUDA(cudaSetDevice(ctx->device));
    FG_CUDA(cudaFree(dptr));
    return FG_OK;
}

fg_status fg_upload(fg_ctx* ctx, void* dst, const void* src, size_t bytes, fg_stream stream) {
    if (!ctx || (!dst && bytes) || (!src && bytes)) return set_error(FG_ERR_INVALID, "null argument");
    if (!bytes) return FG_OK;
    FG_CUDA(cudaSetDevice(ctx->device));
    FG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream_of(ctx, stream)));
    return FG_OK;
}

fg_status fg_download(fg_ctx* ctx, void* dst, const void* src, size_t bytes, fg_stream stream) {
    if (!ctx || (!dst && bytes) || (!src && bytes)) return set_error(FG_ERR_INVALID, "null argument");
    if (!bytes) return FG_OK;
    FG_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = stream_of(ctx, stream);
    FG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
    return fg_sync(ctx, stream);
}

fg_status fg_host_register(fg_ctx* ctx, void* host, size_t bytes) {
    if (!ctx || !host) return set_error(FG_ERR_INVALID, "null argument");
    FG_CUDA(cudaHostRegister(host, bytes, cudaHostRegisterDefault));
    return FG_OK;
}

fg_status fg_host_unregister(fg_ctx* ctx, void* host) {
    if (!ctx || !host) return set_error(FG_ERR_INVALID, "null argument");
    FG_CUDA(cudaHostUnregister(host));
    return FG_OK;
}

fg_status fg_gemm(fg_ctx* ctx, fg_dtype dtype, fg_mode mode, int ozaki_slices, size_t m,
                  size_t n, size_t k, const void* alpha, const void* a, size_t lda,
                  const void* b, size_t ldb, const void* beta, void* c, size_t ldc,
                  int accumulate, fg_stream stream) {
    if (!ctx) return set_error(FG_ERR_INVALID, "null context");
    if (!valid_dtype(dtype)) return set_error(FG_ERR_DTYPE, "unknown dtype");
    if (mode != FG_MODE_PLAIN && mode != FG_MODE_SPLIT && mode != FG_MODE_SPLIT_F16) return set_error(FG_ERR_INVALID, "unknown mode");
    Gemm g;
    g.dtype = dtype;
    g.mode = mode;
    g.slices = ozaki_slices;
    g.M = (long long)m; g.N = (long long)n; g.K = (long long)k;
    g.A = a; g.lda = (long long)lda;
    g.B = b; g.ldb = (long long)ldb;
    g.C = c; g.ldc = (long long)ldc;
    g.accumulate = accumulate;
    set_scalars(g, alpha, beta);
    FG_CUDA(cudaSetDevice(ctx->device));
    return run_gemm(ctx, g, stream_of(ctx, stream));
}

fg_status fg_gemm_f64(fg_ctx* ctx, fg_mode mode, int slices, size_t m, size_t n, size_t k,
                      double alpha, const double* a, const double* b, double beta, double* c,
                      fg_stream stream) {
    return fg_gemm(ctx, FG_F64, mode, slices, m, n, k, &alpha, a, k, b, n, &beta, c, n, 0, stream);
}

fg_status fg_gemm_f32(fg_ctx* ctx, fg_mode mode, size_t m, size_t n, size_t k, float alpha,
                      const float* a, const float* b, float beta, float* c, fg_stream stream) {
    return fg_gemm(ctx, FG_F32, mode, 0, m, n, k, &alpha, a, k, b, n, &beta, c, n, 0, stream);
}

fg_status fg_gemm_c64(fg_ctx* ctx, fg_mode mode, int slices, size_t m, size_t n, size_t k,
                      double ar, double ai, const double* a, const double* b, double br,
                      double bi, double* c, fg_stream stream) {
    double al[2] = {ar, ai}, be[2] = {br, bi};
    return fg_gemm(ctx, FG_C64, mode, slices, m, n, k, al, a, k, b, n, be, c, n, 0, stream);
}

fg_status fg_gemm_c32(fg_ctx* ctx, fg_mode mode, size_t m, size_t n, size_t k, float ar,
                      float ai, const float* a, const float* b, float br, float bi, float* c,
                      fg_stream stream) {
    float al[2] = {ar, ai}, be[2] = {br, bi};
    return fg_gemm(ctx, FG_C32, mode, 0, m, n, k, al, a, k, b, n, be, c, n, 0, stream);
}

fg_status fg_gemm_i8_signed(fg_ctx* ctx, size_t m, size_t n, size_t k, const int8_t* a,
                            const int8_t* b, int32_t* c, int accumulate, fg_stream stream) {
    return fg_gemm(ctx, FG_I8, FG_MODE_PLAIN, 0, m, n, k, nullptr, a, k, b, n, nullptr, c, n,
                   accumulate, stream);
}

fg_status fg_gemm_i8(fg_ctx* ctx, size_t m, size_t n, size_t k, const uint8_t* a,
                     const int8_t* b, int32_t* c, int accumulate, fg_stream stream) {
    return fg_gemm(ctx, FG_U8I8, FG_MODE_PLAIN, 0, m, n, k, nullptr, a, k, b, n, nullptr, c, n,
                   accumulate, stream);
}

fg_status fg_gemm_i16(fg_ctx* ctx, size_t m, size_t n, size_t k, const int16_t* a,
                      const int16_t* b, int32_t* c, int accumulate, fg_stream stream) {
    return fg_gemm(ctx, FG_I16, FG_MODE_PLAIN, 0, m, n, k, nullptr, a, k, b, n, nullptr, c, n,
                   accumulate, stream);
}

fg_status fg_gemm_bf16_f32(fg_ctx* ctx, size_t m, size_t n, size_t k, const uint16_t* a,
                           const uint16_t* b, float* c, int accumulate, fg_stream stream) {
    return fg_gemm(ctx, FG_BF16, FG_MODE_PLAIN, 0, m, n, k, nullptr, a, k, b, n, nullptr, c, n,
                   accumulate, stream);
}

fg_status fg_gemm_f16_f32(fg_ctx* ctx, size_t m, size_t n, size_t k, const uint16_t* a,
                          const uint16_t* b, float* c, int accumulate, fg_stream stream) {
    return fg_gemm(ctx, FG_F16, FG_MODE_PLAIN, 0, m, n, k, nullptr, a, k, b, n, nullptr, c, n,
                   accumulate, stream);
}

fg_status fg_quantized_matmul(fg_ctx* ctx, size_t m, size_t n, size_t k, const uint8_t* a,
                              uint8_t a_zp, float scale_a, const int8_t* b, int8_t b_zp,
                              float scale_b, float* c, int accumulate, fg_stream stream) {
    if (!ctx) return set_error(FG_ERR_INVALID, "null context");
    if (m == 0 || n == 0) return FG_OK;
    if (!c || (k > 0 && (!a || !b))) return set_error(FG_ERR_INVALID, "null operand pointer");
    FG_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = stream_of(ctx, stream);
    if (k == 0) {  // gemm/mod.rs:509-519: zeros, or C untouched when accumulating
        if (!accumulate) {
            FG_CUDA(cudaMemsetAsync(c, 0, m * n * sizeof(float), st));
        }
        return FG_OK;
    }
    return launch_qmm(ctx, (long long)m, (long long)n, (long long)k, a, a_zp, scale_a * scale_b, b,
                      b_zp, c, accumulate, st);
}

// Host-pointer GEMM, pipelined over row panels of A and C: B goes up first,
// then panel i of A (and of C when it is read) on the copy-in stream; the
// GEMM of panel i runs on the compute stream once its inputs have landed and
// its C panel comes back on the copy-out stream while later panels are still
// uploading, so the host<->device copies (full duplex) overlap each other
// and the GEMMs.  Panels are whole 256-row tiles; small problems use one.
fg_status fg_gemm_host(fg_ctx* ctx, fg_dtype dtype, fg_mode mode, int slices, size_t m,
                       size_t n, size_t k, const void* alpha, const void* a, const void* b,
                       const void* beta, void* c, int accumulate) {
    if (!ctx) return set_error(FG_ERR_INVALID, "null context");
    if (!valid_dtype(dtype)) return set_error(FG_ERR_DTYPE, "unknown dtype");
    if (m == 0 || n == 0) return FG_OK;
    if (!c || (k > 0 && (!a || !b))) return set_error(FG_ERR_INVALID, "null operand pointer");
    FG_CUDA(cudaSetDevice(ctx->device));
    std::lock_guard<std::mutex> lk(ctx->host_mu);
    cudaStream_t s_in = ctx->stream, s_cmp = ctx->pipe_comp, s_out = ctx->pipe_out;
    const size_t ein = in_size(dtype), eout = out_size(dtype);
    const size_t ia = ein * m * k, ib = ein * k * n, ic = eout * m * n;
    bool reads_c = accumulate != 0;
    if (!is_integer(dtype) && beta) {
        const double* bd = static_cast<const double*>(beta);
        const float* bf = static_cast<const float*>(beta);
        switch (dtype) {
            case FG_F64: reads_c = bd[0] != 0.0; break;
            case FG_F32: reads_c = bf[0] != 0.0f; break;
            case FG_C64: reads_c = bd[0] != 0.0 || bd[1] != 0.0; break;
            case FG_C32: reads_c = bf[0] != 0.0f || bf[1] != 0.0f; break;
            default: break;
        }
    }
    Scratch sa, sb, sc;
    FG_TRY(sa.alloc(ia, s_in));
    FG_TRY(sb.alloc(ib, s_in));
    FG_TRY(sc.alloc(ic, s_in));
    // Destroyed before the scratch (declared after it): whatever path
    // leaves, the frees queued on s_in wait for the compute and copy-out
    // streams.
    struct Join {
        cudaStream_t in, cmp, out;
        ~Join() {
            for (cudaStream_t s : {cmp, out}) {
                cudaEvent_t e;
                if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) == cudaSuccess) {
                    cudaEventRecord(e, s);
                    cudaStreamWaitEvent(in, e, 0);
                    cudaEventDestroy(e);
                }
            }
        }
    } join{s_in, s_cmp, s_out};
    const size_t total = ia + ib + ic;
    static const size_t kPanelBytes = [] {
        const char* e = getenv("FG_PANEL_MB");
        return static_cast<size_t>(e ? std::max(1, atoi(e)) : 64) << 20;
    }();
    long long panels = total <= kPanelBytes ? 1 : std::min<long long>(32, (total + kPanelBytes - 1) / kPanelBytes);
    long long rows = ((long long)m + panels - 1) / panels;
    rows = (rows + 255) / 256 * 256;
    panels = ((long long)m + rows - 1) / rows;
    if (ib) FG_CUDA(cudaMemcpyAsync(sb.p, b, ib, cudaMemcpyHostToDevice, s_in));
    uint8_t* da = static_cast<uint8_t*>(sa.p);
    uint8_t* dc = static_cast<uint8_t*>(sc.p);
    const uint8_t* ha = static_cast<const uint8_t*>(a);
    uint8_t* hc = static_cast<uint8_t*>(c);
    // The last panel's GEMM and copy-out run after every input has arrived,
    // so the schedule ends on a 256-row piece to keep that tail short.
    std::vector<std::pair<size_t, size_t>> parts;  // (first row, rows)
    for (size_t r0 = 0; r0 < m;) {
        const size_t mi = std::min<size_t>(m - r0, static_cast<size_t>(rows));
        if (panels > 1 && r0 + mi == m && mi > 512) {
            parts.emplace_back(r0, mi - 256);
            parts.emplace_back(r0 + mi - 256, 256);
            break;
        }
        parts.emplace_back(r0, mi);
        r0 += mi;
    }
    for (const auto& part : parts) {
        const size_t r0 = part.first, mi = part.second;
        const size_t oa = r0 * k * ein, na = mi * k * ein, oc = r0 * n * eout, nc = mi * n * eout;
        if (na) FG_CUDA(cudaMemcpyAsync(da + oa, ha + oa, na, cudaMemcpyHostToDevice, s_in));
        if (reads_c) FG_CUDA(cudaMemcpyAsync(dc + oc, hc + oc, nc, cudaMemcpyHostToDevice, s_in));
        cudaEvent_t in_ready, out_ready;
        FG_CUDA(cudaEventCreateWithFlags(&in_ready, cudaEventDisableTiming));
        cudaEventRecord(in_ready, s_in);  // after B and this panel's copies
        cudaStreamWaitEvent(s_cmp, in_ready, 0);
        cudaEventDestroy(in_ready);
        FG_TRY(fg_gemm(ctx, dtype, mode, slices, mi, n, k, alpha, da + oa, k, sb.p, n, beta,
                       dc + oc, n, accumulate, s_cmp));
        FG_CUDA(cudaEventCreateWithFlags(&out_ready, cudaEventDisableTiming));
        cudaEventRecord(out_ready, s_cmp);
        cudaStreamWaitEvent(s_out, out_ready, 0);
        cudaEventDestroy(out_ready);
        FG_CUDA(cudaMemcpyAsync(hc + oc, dc + oc, nc, cudaMemcpyDeviceToHost, s_out));
    }
    FG_CUDA(cudaStreamSynchronize(s_out));
    FG_CUDA(cudaStreamSynchronize(s_cmp));
    return fg_sync(ctx, s_in);
}

fg_status fg_gemm_f64_host(fg_ctx* ctx, fg_mode mode, int slices, size_t m, size_t n, size_t k,
                           double alpha, const double* a, const double* b, double beta,
                           double* c) {
    return fg_gemm_host(ctx, FG_F64, mode, slices, m, n, k, &alpha, a, b, &beta, c, 0);
}

fg_status fg_gemm_f32_host(fg_ctx* ctx, fg_mode mode, size_t m, size_t n, size_t k,
                           float alpha, const float* a, const float* b, float beta, float* c) {
    return fg_gemm_host(ctx, FG_F32, mode, 0, m, n, k, &alpha, a, b, &beta, c, 0);
}

fg_status fg_gemm_batched_strided(fg_ctx* ctx, fg_dtype dtype, fg_mode mode, int slices,
                                  size_t batch, size_t m, size_t n, size_t k, const void* alpha,
                                  const void* a, size_t lda, int64_t stride_a, const void* b,
                                  size_t ldb, int64_t stride_b, const void* beta, void* c,
                                  size_t ldc, int64_t stride_c, int accumulate,
                                  fg_stream stream) {
    if (!ctx) return set_error(FG_ERR_INVALID, "null context");
    if (!valid_dtype(dtype)) return set_error(FG_ERR_DTYPE, "unknown dtype");
    if (batch > INT32_MAX) return set_error(FG_ERR_UNSUPPORTED, "batch too large");
    if (stride_a < 0 || stride_b < 0 || stride_c <= 0 && batch > 1)
        return set_error(FG_ERR_INVALID, "bad batch stride");
    Gemm g;
    g.dtype = dtype;
    g.mode = mode;
    g.slices = slices;
    g.M = (long long)m; g.N = (long long)n; g.K = (long long)k;
    g.A = a; g.lda = (long long)lda;
    g.B = b; g.ldb = (long long)ldb;
    g.C = c; g.ldc = (long long)ldc;
    g.accumulate = accumulate;
    set_scalars(g, alpha, beta);
    g.batch = (int)batch;
    g.bdims = 1;
    g.bshape[0] = (int)std::max<size_t>(batch, 1);
    g.a_count = stride_a ? (long long)batch : 1;
    g.b_count = stride_b ? (long long)batch : 1;
    g.a_istride[0] = stride_a ? 1 : 0;
    g.b_istride[0] = stride_b ? 1 : 0;
    g.a_mstride = stride_a;
    g.b_mstride = stride_b;
    g.c_stride = stride_c;
    FG_CUDA(cudaSetDevice(ctx->device));
    return run_gemm(ctx, g, stream_of(ctx, stream));
}

fg_status fg_matmul(fg_ctx* ctx, fg_dtype dtype, fg_mode mode, const void* a, int ndim_a,
                    const int64_t* shape_a, const void* b, int ndim_b, const int64_t* shape_b,
                    void* c, int64_t* out_shape, int* out_ndim, fg_stream stream) {
    if (!ctx) return set_error(FG_ERR_INVALID, "null context");
    if (!valid_dtype(dtype)) return set_error(FG_ERR_DTYPE, "unknown dtype");
    if (ndim_a < 1 || ndim_b < 1 || !shape_a || !shape_b)
        return set_error(FG_ERR_SHAPE, "matmul: operands must have at least one dimension");
    if (ndim_a == 1 && ndim_b == 1)  // products/mod.rs:371-373
        return set_error(FG_ERR_SHAPE, "matmul: cannot multiply two 1D arrays (use dot instead)");
    for (int i = 0; i < ndim_a; ++i)
        if (shape_a[i] < 0) return set_error(FG_ERR_SHAPE, "negative extent");
    for (int i = 0; i < ndim_b; ++i)
        if (shape_b[i] < 0) return set_error(FG_ERR_SHAPE, "negative extent");
    // Promote 1-D operands (NumPy): a (k,) -> (1, k); b (k,) -> (k, 1).
    std::vector<int64_t> sa(shape_a, shape_a + ndim_a), sb(shape_b, shape_b + ndim_b);
    const bool a_vec = ndim_a == 1, b_vec = ndim_b == 1;
    if (a_vec) sa.insert(sa.begin(), 1);
    if (b_vec) sb.push_back(1);
    const int64_t M = sa[sa.size() - 2], K = sa[sa.size() - 1];
    const int64_t K2 = sb[sb.size() - 2], N = sb[sb.size() - 1];
    if (K != K2)
        return set_error(FG_ERR_SHAPE, "matmul: inner dimensions don't match (" + std::to_string(K) +
                                           " != " + std::to_string(K2) + ")");
    // Broadcast the batch dims (right-aligned), products/mod.rs:661-686
    // semantics but with NumPy indexing for every broadcast pattern.
    const size_t ba = sa.size() - 2, bb = sb.size() - 2, nb = std::max(ba, bb);
    if (nb > 4) return set_error(FG_ERR_UNSUPPORTED, "matmul: more than 4 batch dimensions");
    std::vector<int64_t> bshape(nb);
    for (size_t i = 0; i < nb; ++i) {
        int64_t da = i < nb - ba ? 1 : sa[i - (nb - ba)];
        int64_t db = i < nb - bb ? 1 : sb[i - (nb - bb)];
        if (da == db || db == 1) bshape[i] = da;
        else if (da == 1) bshape[i] = db;
        else return set_error(FG_ERR_BROADCAST, "matmul: batch shapes do not broadcast");
    }
    // Output shape.
    std::vector<int64_t> os(bshape);
    if (!a_vec) os.push_back(M);
    if (!b_vec) os.push_back(N);
    if (out_ndim) *out_ndim = (int)os.size();
    if (out_shape) for (size_t i = 0; i < os.size(); ++i) out_shape[i] = os[i];
    if (!c) return FG_OK;
    Gemm g;
    g.dtype = dtype;
    g.mode = mode;
    g.M = M; g.N = N; g.K = K;
    g.A = a; g.lda = K;
    g.B = b; g.ldb = N;
    g.C = c; g.ldc = N;
    int64_t batch = 1;
    for (auto d : bshape) batch *= d;
    if (batch > INT32_MAX) return set_error(FG_ERR_UNSUPPORTED, "batch too large");
    g.batch = (int)batch;
    g.bdims = (int)nb;
    // matrix-index strides of each operand over the output batch dims
    int64_t acount = 1, bcount = 1;
    for (int i = (int)nb - 1; i >= 0; --i) {
        const size_t ia = (size_t)i, ib = (size_t)i;
        const int64_t da = ia < nb - ba ? 1 : sa[ia - (nb - ba)];
        const int64_t db = ib < nb - bb ? 1 : sb[ib - (nb - bb)];
        g.bshape[i] = (int)bshape[i];
        g.a_istride[i] = da == 1 ? 0 : acount;
        g.b_istride[i] = db == 1 ? 0 : bcount;
        acount *= da;
        bcount *= db;
    }
    g.a_count = acount;
    g.b_count = bcount;
    g.a_mstride = M * K;
    g.b_mstride = K * N;
    g.c_stride = M * N;
    if (g.bdims == 0) { g.bdims = 1; g.bshape[0] = 1; }
    FG_CUDA(cudaSetDevice(ctx->device));
    return run_gemm(ctx, g, stream_of(ctx, stream));
}

}  // extern "C"
