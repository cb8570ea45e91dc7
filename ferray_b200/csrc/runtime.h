// runtime.h -- host-side internals shared by the C-ABI translation units:
// the context, error plumbing, scratch allocation and the internal GEMM
// problem description every entry point lowers to.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/ferray_gpu.h"
#include "fg_device.cuh"

struct fg_ctx {
    int device = 0;
    int sm_count = 0;
    int cc_major = 0, cc_minor = 0;
    size_t hbm_bytes = 0;
    cudaStream_t stream = nullptr;
    // host-pointer calls: GEMMs and copy-out run on their own streams so the
    // copies of one row panel overlap the GEMM of another
    cudaStream_t pipe_comp = nullptr, pipe_out = nullptr;
    fg::DevStatus* d_status = nullptr;  // kernel error word (device)
    std::mutex mu;
    std::mutex host_mu;  // one pipelined host-pointer call at a time
};

namespace fgrt {

extern std::atomic<uint64_t> g_launches;

fg_status set_error(fg_status s, const std::string& msg);
fg_status cuda_error(cudaError_t e, const char* what);

#define FG_CUDA(call)                                         \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) return fgrt::cuda_error(e_, #call); \
    } while (0)

#define FG_TRY(call)                      \
    do {                                  \
        fg_status s_ = (call);            \
        if (s_ != FG_OK) return s_;       \
    } while (0)

inline cudaStream_t stream_of(fg_ctx* ctx, fg_stream s) {
    return s ? static_cast<cudaStream_t>(s) : ctx->stream;
}

inline void count_launch(uint64_t n = 1) { g_launches.fetch_add(n, std::memory_order_relaxed); }

// Optional per-family kernel timing (fg_profile_enable).  Usage:
//   ProfScope ps("family", stream); launch<<<...>>>; ps.stop();
extern std::atomic<int> g_prof_on;
void prof_record(const char* family, cudaEvent_t start, cudaEvent_t stop);
struct ProfScope {
    const char* fam;
    cudaStream_t st;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    ProfScope(const char* family, cudaStream_t stream) : fam(family), st(stream) {
        if (g_prof_on.load(std::memory_order_relaxed)) {
            cudaEventCreate(&e0);
            cudaEventCreate(&e1);
            cudaEventRecord(e0, st);
        }
    }
    void stop() {
        if (e0) {
            cudaEventRecord(e1, st);
            prof_record(fam, e0, e1);
            e0 = e1 = nullptr;
        }
    }
    ~ProfScope() { stop(); }
};

// Stream-ordered scratch: freed on the same stream after the kernels that
// use it, so concurrent calls on other streams never share it.
struct Scratch {
    void* p = nullptr;
    cudaStream_t st = nullptr;
    Scratch() = default;
    Scratch(const Scratch&) = delete;
    Scratch& operator=(const Scratch&) = delete;
    fg_status alloc(size_t bytes, cudaStream_t stream) {
        st = stream;
        if (bytes == 0) bytes = 16;
        cudaError_t e = cudaMallocAsync(&p, bytes, stream);
        if (e != cudaSuccess) {
            p = nullptr;
            cudaGetLastError();
            return set_error(FG_ERR_OOM, "scratch allocation of " + std::to_string(bytes) + " bytes failed");
        }
        return FG_OK;
    }
    ~Scratch() {
        if (p) cudaFreeAsync(p, st);
    }
};

// Element size of the operands / result of a dtype.
inline size_t in_size(fg_dtype d) {
    switch (d) {
        case FG_F64: return 8;
        case FG_F32: return 4;
        case FG_C64: return 16;
        case FG_C32: return 8;
        case FG_I8: case FG_U8I8: return 1;
        case FG_I16: return 2;
        case FG_BF16: case FG_F16: return 2;
    }
    return 0;
}
inline size_t out_size(fg_dtype d) {
    switch (d) {
        case FG_I8: case FG_U8I8: case FG_I16: return 4;
        case FG_BF16: case FG_F16: return 4;
        default: return in_size(d);
    }
}
inline bool is_complex(fg_dtype d) { return d == FG_C64 || d == FG_C32; }
inline bool is_integer(fg_dtype d) { return d == FG_I8 || d == FG_U8I8 || d == FG_I16; }
// 16-bit float operands, f32 result, accumulate-flag semantics like the integers.
inline bool is_half(fg_dtype d) { return d == FG_BF16 || d == FG_F16; }

// One (possibly batched, possibly broadcast) GEMM after argument lowering.
struct Gemm {
    fg_dtype dtype = FG_F64;
    fg_mode mode = FG_MODE_PLAIN;
    int slices = 0;
    long long M = 0, N = 0, K = 0;
    const void* A = nullptr;
    long long lda = 0;
    const void* B = nullptr;
    long long ldb = 0;
    void* C = nullptr;
    long long ldc = 0;
    // batch: `batch` output matrices C + i*c_stride; operand matrix of output
    // i decomposes i over bshape and dots with a_istride/b_istride (matrix
    // indices), matrices a_mstride / b_mstride elements apart.
    int batch = 1;
    int bdims = 0;
    int bshape[4] = {1, 1, 1, 1};
    long long a_istride[4] = {0, 0, 0, 0}, b_istride[4] = {0, 0, 0, 0};
    long long a_count = 1, b_count = 1;       // distinct operand matrices
    long long a_mstride = 0, b_mstride = 0;   // elements between operand matrices
    long long c_stride = 0;
    double alpha_re = 1, alpha_im = 0, beta_re = 0, beta_im = 0;
    int accumulate = 0;
};

fg_status run_gemm(fg_ctx* ctx, const Gemm& g, cudaStream_t st);

// Family launchers (gemm_tc.cu, gemm_simt.cu, gemm_ozaki.cu).
fg_status launch_simt(fg_ctx* ctx, const Gemm& g, cudaStream_t st);
fg_status launch_int_tc(fg_ctx* ctx, const Gemm& g, cudaStream_t st);
fg_status launch_half_tc(fg_ctx* ctx, const Gemm& g, cudaStream_t st);
fg_status launch_split_bf16(fg_ctx* ctx, const Gemm& g, cudaStream_t st);
fg_status launch_ozaki(fg_ctx* ctx, const Gemm& g, cudaStream_t st);
fg_status launch_qmm(fg_ctx* ctx, long long M, long long N, long long K, const uint8_t* a,
                     int a_zp, float scale, const int8_t* b, int b_zp, float* c,
                     int accumulate, cudaStream_t st);

// Grouped batches in device form (grouped.cu): build (host layout) ->
// bind (device base + host staging image) -> launch (async upload + kernels).
struct GroupedJob;
GroupedJob* grouped_job_new();
void grouped_job_free(GroupedJob* j);
fg_status grouped_job_build(fg_ctx* ctx, fg_dtype dtype, fg_mode mode, const fg_problem* table,
                            size_t count, GroupedJob* j);
size_t grouped_job_dev_bytes(const GroupedJob* j);
size_t grouped_job_host_bytes(const GroupedJob* j);
fg_status grouped_job_bind(GroupedJob* j, void* dev_base, void* host_stage);
fg_status grouped_job_launch(GroupedJob* j, cudaStream_t st);

// cuTensorMapEncodeTiled through the runtime's driver entry point (no
// link-time dependency on libcuda).
fg_status encode_map(CUtensorMap* map, CUtensorMapDataType dt, int rank, const void* base,
                     const uint64_t* dims, const uint64_t* strides_bytes, const uint32_t* box);

}  // namespace fgrt
