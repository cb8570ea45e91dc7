/*
 * ferray_gpu.h -- C ABI of the ferray B200 GEMM backend (libferray_b200.so).
 *
 * Replaces the GEMM behind ferray_linalg::matmul / ferray::matmul.  Every
 * entry point below names the ferray function (file:line inside the ferray
 * workspace) whose contract it keeps.  Conventions:
 *
 *  - Matrices are row-major.  Leading dimensions are in ELEMENTS (complex
 *    elements for complex types), exactly like the reference's internal
 *    drivers (gemm/outer.rs: lda, ldb, ldc); the fg_gemm_<dtype> forms fix
 *    lda = k, ldb = n, ldc = n like the reference's public entry points.
 *  - Complex operands are interleaved (re, im) pairs, the layout of
 *    num_complex::Complex<T> (repr(C)).  As in ferray, "c64" means
 *    Complex<f64> and "c32" means Complex<f32>.
 *  - Pointers passed to fg_gemm_* / fg_matmul_* are DEVICE pointers (from
 *    fg_buffer_alloc or any cudaMalloc'd memory of the context's device).
 *    The *_host forms take host pointers, stage through the device and
 *    return when the result is back in host memory: they are the drop-in
 *    for ferray's slice-based entry points.
 *  - Every function returns fg_status.  FG_OK is 0.  The reference returns
 *    `false` when no CPU kernel applies and FerrayError::ShapeMismatch /
 *    BroadcastFailure for bad shapes (ferray-core/src/error.rs:16-99); here
 *    those become FG_ERR_UNSUPPORTED, FG_ERR_SHAPE and FG_ERR_BROADCAST.
 *  - Device-pointer calls are asynchronous on `stream` (NULL = the
 *    context's stream).  Kernel-side failures (a bounded wait that ran out)
 *    are reported by the next fg_sync on that context.
 *  - Thread safety: a context may be used from many host threads; calls on
 *    different streams may overlap on the device.  Scratch memory comes
 *    from the stream-ordered allocator on the call's stream.
 *  - No CPU fallback: without a usable sm_100 device fg_init fails.
 */
#ifndef FERRAY_GPU_H
#define FERRAY_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum fg_status {
    FG_OK = 0,
    FG_ERR_SHAPE = 1,       /* inner dimensions / lengths disagree            */
    FG_ERR_DTYPE = 2,       /* dtype not valid for this entry point           */
    FG_ERR_OOM = 3,         /* device allocation failed                        */
    FG_ERR_BUDGET = 4,      /* request exceeds the server's HBM budget        */
    FG_ERR_TIMEOUT = 5,     /* a bounded device or host wait ran out           */
    FG_ERR_DEVICE = 6,      /* CUDA error                                      */
    FG_ERR_INVALID = 7,     /* bad argument (null pointer, bad mode, ...)      */
    FG_ERR_UNSUPPORTED = 8, /* no kernel for this case (reference: `false`)    */
    FG_ERR_BROADCAST = 9    /* batch shapes do not broadcast                   */
} fg_status;

typedef enum fg_dtype {
    FG_F64 = 0,  /* f64                     */
    FG_F32 = 1,  /* f32                     */
    FG_C64 = 2,  /* Complex<f64> (16 bytes) */
    FG_C32 = 3,  /* Complex<f32> (8 bytes)  */
    FG_I8 = 4,   /* i8 x i8 -> i32          */
    FG_U8I8 = 5, /* u8 x i8 -> i32          */
    FG_I16 = 6,  /* i16 x i16 -> i32        */
    FG_BF16 = 7, /* bf16 x bf16 -> f32 (raw 16-bit patterns) */
    FG_F16 = 8   /* f16 x f16 -> f32 (IEEE binary16)         */
} fg_dtype;

typedef enum fg_mode {
    /* f64/c64: FP64 pipe; f32/c32: FFMA; integers: integer tensor cores.   */
    FG_MODE_PLAIN = 0,
    /* f32/c32: 3 x BF16 products on tcgen05 with FP32 accumulation;        */
    /* f64/c64: Ozaki INT8 slicing with exact INT32 accumulation.           */
    /* Integer dtypes ignore the mode (they are exact either way).          */
    FG_MODE_SPLIT = 1,
    /* f32/c32: 3 products (hi*hi + hi*lo + lo*hi) of two FP16 slices of    */
    /* the operands scaled by powers of two from their largest magnitudes,  */
    /* on tcgen05 with FP32 accumulation: about 23 bits per operand against */
    /* 17 for two BF16 slices, at the same tensor-core rate.  Grouped      */
    /* launches (ragged batches, the server's folded small requests) run it */
    /* as FG_MODE_SPLIT; f64/c64 and integer dtypes treat it as             */
    /* FG_MODE_SPLIT.  No reference counterpart.                            */
    FG_MODE_SPLIT_F16 = 2
} fg_mode;

typedef struct fg_ctx fg_ctx;
typedef void *fg_stream; /* a cudaStream_t */

/* ------------------------------------------------------------ context */
/* Opens `device` (must be sm_100).  ferray's GEMM has no handle; its pool
 * is process-global (gemm/outer.rs:142-155). */
fg_status fg_init(int device, fg_ctx **out);
fg_status fg_shutdown(fg_ctx *ctx);
/* Waits for `stream` (NULL: context stream) and reports kernel-side errors
 * recorded since the last fg_sync. */
fg_status fg_sync(fg_ctx *ctx, fg_stream stream);
const char *fg_status_string(fg_status s);
/* Message of the last error raised on the calling thread ("" if none). */
const char *fg_last_error(void);
/* Number of kernels this library has launched in the process. */
uint64_t fg_launch_count(void);
/* Kernel timing for roofline bookkeeping (no reference counterpart; ferray
 * has no tracing).  While enabled, every main GEMM kernel launch is
 * bracketed by CUDA events on its own stream; fg_profile_collect waits for
 * them and returns per-kernel-family launch counts and summed device time,
 * then clears the records. */
typedef struct fg_profile_entry {
    char name[48];
    uint64_t launches;
    double total_ms;
} fg_profile_entry;
fg_status fg_profile_enable(int on);
fg_status fg_profile_collect(fg_profile_entry *out, int capacity, int *count);
/* Measured dense throughput of one compute pipe of this GPU, for roofline
 * fractions against a measured rather than a spec-sheet peak (no reference
 * counterpart).  A persistent grid keeps the pipe busy on on-chip data for
 * about 10 ms: INT8 and BF16 as tcgen05.mma (M 128, N 256) from shared
 * memory into TMEM, FP64 as DMMA (mma.sync m8n8k4) and FP32 as FFMA on
 * registers.  *per_second: ops (2 per multiply-add) per second. */
typedef enum fg_probe_pipe {
    FG_PROBE_INT8 = 0,
    FG_PROBE_BF16 = 1,
    FG_PROBE_FP64 = 2,
    FG_PROBE_FFMA = 3
} fg_probe_pipe;
fg_status fg_probe_peak(fg_ctx *ctx, int which, double *per_second);
/* Device properties used for roofline bookkeeping. */
fg_status fg_device_info(fg_ctx *ctx, int *sm_count, int *cc_major, int *cc_minor,
                         size_t *hbm_bytes);

/* Failure-detection self test: launches one kernel whose bounded device
 * wait nothing satisfies; it gives up after `timeout_us` (1 us .. 1 s), so
 * the next fg_sync returns FG_ERR_TIMEOUT and the context stays usable.
 * The same bounded wait guards every pipeline barrier of the GEMM kernels. */
fg_status fg_selftest_wait_timeout(fg_ctx *ctx, uint32_t timeout_us, fg_stream stream);

/* ------------------------------------------------------------ .npy ingest */
/* Parses an .npy byte image (format 1.0 / 2.0 / 3.0, the header rules of
 * ferray-io/src/npy/header.rs:32-106; host only, no device needed): element
 * type as the fg_dtype of a GEMM operand (<f8 F64, <f4 F32, <c16 C64, <c8 C32,
 * |i1 I8, |u1 U8I8 (the u8 operand), <i2 I16, <f2 F16), shape (up to 8
 * dims), Fortran order flag and the payload offset.  FG_ERR_DTYPE for other
 * or big-endian descrs, FG_ERR_SHAPE when the payload is shorter than the
 * shape, FG_ERR_INVALID for a malformed image. */
fg_status fg_npy_parse(const void *bytes, size_t len, fg_dtype *dtype, int64_t *shape, int *ndim,
                       int *fortran_order, size_t *data_offset);
/* Parses the image and copies its payload into a new device buffer
 * (fg_buffer_alloc; free with fg_buffer_free), asynchronously on `stream`
 * (the host bytes must stay valid until the stream reaches the copy).
 * Row-major (C order) only. */
fg_status fg_npy_upload(fg_ctx *ctx, const void *bytes, size_t len, void **dptr, fg_dtype *dtype,
                        int64_t *shape, int *ndim, fg_stream stream);

/* .npz archives held in memory (ferray-io/src/npz/mod.rs:88-200, NpzFile):
 * member names are the archive's file names without a trailing ".npy";
 * a name is fetched from the member "<name>.npy".  Stored and deflate
 * members, ZIP64 archives; every member's CRC-32 is checked.  Host only,
 * except fg_npz_upload. */
fg_status fg_npz_count(const void *bytes, size_t len, size_t *count);
/* Name of member `index` (NUL-terminated into out[cap]; out may be null to
 * ask for *name_len only). */
fg_status fg_npz_name(const void *bytes, size_t len, size_t index, char *out, size_t cap,
                      size_t *name_len);
/* The .npy bytes of array `name` (inflated) into out[cap]; out may be null
 * to ask for *size only.  FG_ERR_INVALID when the name is not listed. */
fg_status fg_npz_read(const void *bytes, size_t len, const char *name, void *out, size_t cap,
                      size_t *size);
/* Array `name` into a new device buffer, as fg_npy_upload (stored members
 * are copied straight from `bytes`). */
fg_status fg_npz_upload(fg_ctx *ctx, const void *bytes, size_t len, const char *name, void **dptr,
                        fg_dtype *dtype, int64_t *shape, int *ndim, fg_stream stream);

/* ------------------------------------------------------------ GEMM chains */
/* multi_dot (products/mod.rs:776-902): mats[i] is a contiguous row-major
 * dims[i] x dims[i+1] device matrix (a 1-D first / last operand is passed as
 * 1 x n / n x 1, as the reference forms its dims), out is dims[0] x
 * dims[count].  The product order is the reference's optimal
 * parenthesisation (same dynamic programme, same tie-breaking); the
 * intermediates stay on the device.  Errors: FG_ERR_INVALID for fewer than 2
 * matrices, FG_ERR_SHAPE for non-positive dims. */
fg_status fg_multi_dot(fg_ctx *ctx, fg_dtype dtype, fg_mode mode, size_t count,
                       const void *const *mats, const int64_t *dims, void *out, fg_stream stream);
/* The parenthesisation fg_multi_dot uses (host only): split[i*count + j] is
 * the k at which the product of matrices i..j is split. */
fg_status fg_multi_dot_order(size_t count, const int64_t *dims, size_t *split);
/* numpy-style tensordot (products/tensordot.rs:35-153): contracts axes_a[i]
 * of `a` with axes_b[i] of `b` (naxes pairs; the scalar form axes = N is
 * the last N of a with the first N of b); out (contiguous) gets a's free
 * axes then b's.  Operands are permuted on the device (free axes first for
 * a, contracted first for b; skipped when already in that order) and
 * contracted by one GEMM.  out_shape receives up to ndim_a + ndim_b dims. */
fg_status fg_tensordot(fg_ctx *ctx, fg_dtype dtype, fg_mode mode, const void *a, int ndim_a,
                       const int64_t *shape_a, const void *b, int ndim_b, const int64_t *shape_b,
                       int naxes, const int *axes_a, const int *axes_b, void *out,
                       int64_t *out_shape, int *out_ndim, fg_stream stream);
/* Two-operand einsum ("ij,jk->ik", "bij,bjk->bik", "ijk,kjl->il", ...;
 * letter labels, implicit output = labels seen once in ASCII order).  Covers
 * the reference's matmul shortcut (products/einsum/mod.rs:251-282) and every
 * pairwise contraction without repeated labels inside one operand
 * (FG_ERR_UNSUPPORTED otherwise, e.g. traces or ellipsis): operands permuted
 * on the device to [batch, free, contracted], one batched GEMM, and the
 * output permuted to the requested order.  out_shape gets up to 8 dims. */
fg_status fg_einsum(fg_ctx *ctx, fg_dtype dtype, fg_mode mode, const char *subscripts,
                    const void *a, int ndim_a, const int64_t *shape_a, const void *b, int ndim_b,
                    const int64_t *shape_b, void *out, int64_t *out_shape, int *out_ndim,
                    fg_stream stream);
/* A^exponent for a square n x n device matrix (solve.rs:456-494): identity
 * for 0, exponentiation by squaring in the reference's order for > 0;
 * negative powers need inv(A) and return FG_ERR_UNSUPPORTED. */
fg_status fg_matrix_power(fg_ctx *ctx, fg_dtype dtype, fg_mode mode, size_t n, const void *a,
                          int64_t exponent, void *out, fg_stream stream);
/* Left-side triangular solve op(A) X = alpha B, in place on the device
 * matrix B (m x n, row stride ldb >= n); A is m x m with row stride
 * lda >= m, lower (upper = 0) or upper triangular, its diagonal taken as 1
 * when unit_diag.  Replaces trsm_left_lower_f64 / trsm_left_upper_f64 /
 * trsm_left_lower_f32 / trsm_left_upper_f32 (ferray-linalg/src/trsm.rs:
 * 46-133): alpha is a host double / float (null = 1); the same block
 * recursion; sub-problems of <= 128 rows are solved with the reference's own
 * operations in its order (bit-identical results), and each trailing update
 * above them, B2 -= L21 X1 (B1 -= U12 X2), is one tuned GEMM in `mode` (f64
 * split: the Ozaki form for updates of at least 4096 in rows, k and n,
 * plain FP64 below).
 * m == 0 or n == 0 returns FG_OK with B untouched.  FG_ERR_DTYPE for dtypes
 * other than f64 / f32. */
fg_status fg_trsm_left(fg_ctx *ctx, fg_dtype dtype, fg_mode mode, int upper, int unit_diag,
                       size_t m, size_t n, const void *alpha, const void *a, size_t lda, void *b,
                       size_t ldb, fg_stream stream);

/* ------------------------------------------------------------ autotune */
/* Tile variant and split-K count per GEMM family come from a table indexed
 * by the size buckets of m, n, k (<=16, <=32, ..., <=4096, >4096), written
 * by ferray_b200/autotune.py from timings on a B200 and compiled in.  The
 * reference's blocking is fixed constants (MC 64, KC 256, NC 512,
 * gemm/outer.rs:66-68); this table is what replaces them. */
typedef enum fg_tune_op {
    FG_TUNE_I8 = 0,        /* i8 x i8 / u8 x i8 -> i32 (tensor cores)       */
    FG_TUNE_SPLIT_F32 = 1, /* 3xBF16 split SGEMM (tensor cores)             */
    FG_TUNE_F64 = 2,       /* plain DGEMM (FP64 pipe)                       */
    FG_TUNE_F32 = 3        /* plain SGEMM (FFMA)                            */
} fg_tune_op;
/* The (variant, splits) the dispatch uses for a problem of this size. */
fg_status fg_tune_lookup(int op, size_t m, size_t n, size_t k, int *variant, int *splits);
/* Forces (variant, splits) for every later call of `op`, process-wide;
 * variant < 0 returns to the table.  For the tuner, not for serving. */
fg_status fg_tune_force(int op, int variant, int splits);
/* Number of kernel variants of `op`. */
fg_status fg_tune_variants(int op, int *count);

/* ------------------------------------------------------------ buffers */
/* Device-resident buffers: the device counterpart of ferray-core's
 * Array storage (ferray-core/src/array/owned.rs:21, buffer.rs:25-49). */
fg_status fg_buffer_alloc(fg_ctx *ctx, size_t bytes, void **dptr);
fg_status fg_buffer_free(fg_ctx *ctx, void *dptr);
fg_status fg_upload(fg_ctx *ctx, void *dst_dev, const void *src_host, size_t bytes,
                    fg_stream stream);
fg_status fg_download(fg_ctx *ctx, void *dst_host, const void *src_dev, size_t bytes,
                      fg_stream stream);
/* Page-lock host memory so uploads/downloads run at full PCIe speed. */
fg_status fg_host_register(fg_ctx *ctx, void *host, size_t bytes);
fg_status fg_host_unregister(fg_ctx *ctx, void *host);

/* ------------------------------------------------------------ raw GEMMs */
/* C = alpha*A@B + beta*C, f64.  Replaces gemm_f64 (gemm/mod.rs:197-328).
 * mode SPLIT = Ozaki INT8: `ozaki_slices` 3..10 = scheme I digit slices,
 * 12..20 = scheme II moduli, 0 = scheme II with 16 moduli (see fg_gemm). */
fg_status fg_gemm_f64(fg_ctx *ctx, fg_mode mode, int ozaki_slices, size_t m, size_t n,
                      size_t k, double alpha, const double *a, const double *b, double beta,
                      double *c, fg_stream stream);
/* C = alpha*A@B + beta*C, f32.  Replaces gemm_f32 (gemm/mod.rs:940-1062).
 * mode SPLIT = 3 x BF16 on tcgen05; SPLIT_F16 = 3 x FP16 of scaled operands. */
fg_status fg_gemm_f32(fg_ctx *ctx, fg_mode mode, size_t m, size_t n, size_t k, float alpha,
                      const float *a, const float *b, float beta, float *c, fg_stream stream);
/* Complex<f64>.  Replaces gemm_c64 (gemm/mod.rs:757-826). */
fg_status fg_gemm_c64(fg_ctx *ctx, fg_mode mode, int ozaki_slices, size_t m, size_t n,
                      size_t k, double alpha_re, double alpha_im, const double *a,
                      const double *b, double beta_re, double beta_im, double *c,
                      fg_stream stream);
/* Complex<f32>.  Replaces gemm_c32 (gemm/mod.rs:669-736). */
fg_status fg_gemm_c32(fg_ctx *ctx, fg_mode mode, size_t m, size_t n, size_t k, float alpha_re,
                      float alpha_im, const float *a, const float *b, float beta_re,
                      float beta_im, float *c, fg_stream stream);
/* i8 x i8 -> i32, wrapping, optional accumulate into C.
 * Replaces gemm_i8_signed (gemm/mod.rs:414-448). */
fg_status fg_gemm_i8_signed(fg_ctx *ctx, size_t m, size_t n, size_t k, const int8_t *a,
                            const int8_t *b, int32_t *c, int accumulate, fg_stream stream);
/* u8 x i8 -> i32, exact (the VNNI semantics).  Replaces gemm_i8
 * (gemm/mod.rs:601-651). */
fg_status fg_gemm_i8(fg_ctx *ctx, size_t m, size_t n, size_t k, const uint8_t *a,
                     const int8_t *b, int32_t *c, int accumulate, fg_stream stream);
/* i16 x i16 -> i32, wrapping.  Replaces gemm_i16 (gemm/mod.rs:348-392). */
fg_status fg_gemm_i16(fg_ctx *ctx, size_t m, size_t n, size_t k, const int16_t *a,
                      const int16_t *b, int32_t *c, int accumulate, fg_stream stream);
/* C = A@B (C += A@B when accumulate), bf16 x bf16 -> f32, on tcgen05
 * kind::f16 with FP32 accumulation straight from the 16-bit operands.
 * Replaces gemm_bf16_f32 (gemm/mod.rs:851-882; ferray widens to f32 and runs
 * its SGEMM).  a, b hold bf16 bit patterns. */
fg_status fg_gemm_bf16_f32(fg_ctx *ctx, size_t m, size_t n, size_t k, const uint16_t *a,
                           const uint16_t *b, float *c, int accumulate, fg_stream stream);
/* Same for IEEE f16 operands.  Replaces gemm_f16_f32 (gemm/mod.rs:906-933). */
fg_status fg_gemm_f16_f32(fg_ctx *ctx, size_t m, size_t n, size_t k, const uint16_t *a,
                          const uint16_t *b, float *c, int accumulate, fg_stream stream);
/* scale_a*scale_b*sum((a-a_zp)*(b-b_zp)) -> f32, zero points and scale fused
 * into the i8 kernel's epilogue.  Replaces quantized_matmul
 * (gemm/mod.rs:484-575). */
fg_status fg_quantized_matmul(fg_ctx *ctx, size_t m, size_t n, size_t k, const uint8_t *a,
                              uint8_t a_zp, float scale_a, const int8_t *b, int8_t b_zp,
                              float scale_b, float *c, int accumulate, fg_stream stream);

/* quantized_matmul that allocates nothing -- no counterpart in the
 * reference.  Same contract and results as fg_quantized_matmul, for callers
 * that may not allocate device memory at call time (memory owned by another
 * allocator, a fixed HBM budget, latency-critical loops).  Its zero-point
 * row/column sums live in one fixed 512 KiB device array per GPU, held until
 * the process exits; the first call on a device looks up that array's
 * address and should come before any stream capture.  Calls share the array,
 * so calls that overlap on the GPU race.  Limits: m, n, k <= 65536; k and n
 * multiples of 16 and a, b 16-byte aligned; otherwise FG_ERR_UNSUPPORTED. */
fg_status fg_quantized_matmul_noalloc(fg_ctx *ctx, size_t m, size_t n, size_t k,
                                      const uint8_t *a, uint8_t a_zp, float scale_a,
                                      const int8_t *b, int8_t b_zp, float scale_b, float *c,
                                      int accumulate, fg_stream stream);

/* Generic strided form of all of the above (the reference's internal
 * drivers take lda/ldb/ldc: gemm/outer.rs:198-210).  `ozaki_slices` in split
 * mode: f64/c64, 3..10 = Ozaki scheme I with that many INT8 digit slices per
 * operand (S(S+1)/2 slice products), 12..20 = Ozaki scheme II with that
 * many moduli (one INT8 product per modulus, Chinese-remainder
 * reconstruction; K up to 130944, longer K runs scheme I with 9 slices),
 * 0 = scheme II with 16 moduli; f32/c32, BF16 slices per operand,
 * 2 (three products, the default for 0) or 3 (six products, exact slicing of
 * f32, for FP32-level accuracy at half the speed).  alpha/beta point to a
 * scalar of the dtype's real type (two for complex: re, im); integer dtypes
 * ignore them and use `accumulate`. */
fg_status fg_gemm(fg_ctx *ctx, fg_dtype dtype, fg_mode mode, int ozaki_slices, size_t m,
                  size_t n, size_t k, const void *alpha, const void *a, size_t lda,
                  const void *b, size_t ldb, const void *beta, void *c, size_t ldc,
                  int accumulate, fg_stream stream);

/* Host-pointer drop-ins: same contracts as the device forms above, with
 * host slices in and out (the signatures of gemm/mod.rs).  Synchronous. */
fg_status fg_gemm_f64_host(fg_ctx *ctx, fg_mode mode, int ozaki_slices, size_t m, size_t n,
                           size_t k, double alpha, const double *a, const double *b,
                           double beta, double *c);
fg_status fg_gemm_f32_host(fg_ctx *ctx, fg_mode mode, size_t m, size_t n, size_t k,
                           float alpha, const float *a, const float *b, float beta, float *c);
fg_status fg_gemm_host(fg_ctx *ctx, fg_dtype dtype, fg_mode mode, int ozaki_slices, size_t m,
                       size_t n, size_t k, const void *alpha, const void *a, const void *b,
                       const void *beta, void *c, int accumulate);

/* ------------------------------------------------------------ batches */
/* Stacked GEMM with one M,N,K for all `batch` problems: problem i reads
 * A + i*stride_a, B + i*stride_b and writes C + i*stride_c (element
 * strides; 0 broadcasts one operand).  Replaces the per-problem loop of
 * matmul_batched (products/mod.rs:579-659). */
fg_status fg_gemm_batched_strided(fg_ctx *ctx, fg_dtype dtype, fg_mode mode, int ozaki_slices,
                                  size_t batch, size_t m, size_t n, size_t k, const void *alpha,
                                  const void *a, size_t lda, int64_t stride_a, const void *b,
                                  size_t ldb, int64_t stride_b, const void *beta, void *c,
                                  size_t ldc, int64_t stride_c, int accumulate,
                                  fg_stream stream);

/* NumPy `matmul` on device arrays of any rank (1-D operands promoted and
 * squeezed, batch dims broadcast with NumPy rules).  Replaces matmul
 * (products/mod.rs:362-437), matmul_batched + broadcast_shapes
 * (:579-686) and matmul_complex (complex.rs:136-264).  The output shape is
 * written to out_shape/out_ndim (capacity 8); pass c = NULL to query it. */
fg_status fg_matmul(fg_ctx *ctx, fg_dtype dtype, fg_mode mode, const void *a, int ndim_a,
                    const int64_t *shape_a, const void *b, int ndim_b, const int64_t *shape_b,
                    void *c, int64_t *out_shape, int *out_ndim, fg_stream stream);

/* Ragged batch: `count` independent problems with their own M, N, K,
 * pointers and leading dimensions, run by ONE persistent grouped kernel
 * driven by a device-side problem table and tile counter.  No reference
 * counterpart (ferray calls matmul_raw once per problem). */
typedef struct fg_problem {
    int64_t m, n, k;
    const void *a;
    const void *b;
    void *c;
    int64_t lda, ldb, ldc;
} fg_problem;

/* `table` is a HOST array; it is copied to the device on `stream`.
 * dtype: FG_F32 (plain FFMA or SPLIT 3xBF16) or FG_I8 (exact). */
fg_status fg_gemm_grouped(fg_ctx *ctx, fg_dtype dtype, fg_mode mode, const fg_problem *table,
                          size_t count, fg_stream stream);

/* Opaque prepared plan for a grouped batch whose shapes repeat: the table is
 * uploaded once and the launch sequence is captured in a CUDA graph;
 * fg_grouped_plan_run replays it. */
typedef struct fg_grouped_plan fg_grouped_plan;
fg_status fg_grouped_plan_create(fg_ctx *ctx, fg_dtype dtype, fg_mode mode,
                                 const fg_problem *table, size_t count, fg_stream stream,
                                 fg_grouped_plan **out);
fg_status fg_grouped_plan_run(fg_grouped_plan *plan, fg_stream stream);
fg_status fg_grouped_plan_destroy(fg_grouped_plan *plan);

/* ------------------------------------------------------------ sharding */
/* Multi-GPU runs are one process per GPU; independent problems (a ragged
 * batch) and requests (a served stream) are split across the processes
 * with no exchange: every rank computes the same assignment from the same
 * list.  ferray's counterpart is the rayon split of a stacked matmul's batch
 * inside one process (products/mod.rs:625-638). */
typedef enum fg_shard_policy {
    FG_SHARD_LPT = 0,    /* heaviest unit first, each to the least-loaded rank */
    FG_SHARD_ONLINE = 1  /* arrival order, each to the least-loaded rank       */
} fg_shard_policy;
/* Indices (ascending) of the units rank `rank` of `world` runs.  `dims` is
 * count x 3 (m, n, k) int64; a unit costs weight[i] when `weight` is not
 * NULL, else 2mnk.  Ties go to the lower rank.  `out` holds up to `count`. */
fg_status fg_shard_plan(const int64_t *dims, const double *weight, size_t count, int world,
                        int rank, int policy, int64_t *out, size_t *out_count);
/* fg_gemm_grouped over this rank's FG_SHARD_LPT shard of `table`. */
fg_status fg_gemm_grouped_shard(fg_ctx *ctx, fg_dtype dtype, fg_mode mode,
                                const fg_problem *table, size_t count, int world, int rank,
                                fg_stream stream);

/* ------------------------------------------------------------ serving */
/* Continuous-batching request loop.  Host threads submit matmul requests
 * (mixed shapes and dtypes) whose operands are already on the device; the
 * server admits them against an HBM budget, folds queued requests into
 * grouped launches while earlier ones still run on other streams, and
 * completes tickets as their results land.  No reference counterpart. */
typedef struct fg_server fg_server;

typedef struct fg_request {
    fg_dtype dtype;
    fg_mode mode;
    int64_t m, n, k;
    const void *a; /* device, row-major m x k  */
    const void *b; /* device, row-major k x n  */
    void *c;       /* device, row-major m x n  */
    size_t scratch_bytes; /* 0: the server estimates it from the shape */
} fg_request;

typedef struct fg_server_stats {
    uint64_t completed;
    uint64_t launches;
    uint64_t grouped_launches;
    double p50_ms, p99_ms, mean_ms;
    double useful_flops;   /* sum of 2mnk (8mnk complex) of completed work */
    double busy_seconds;   /* wall time from first admit to last completion */
    size_t hbm_in_use, hbm_peak;
} fg_server_stats;

fg_status fg_server_start(fg_ctx *ctx, size_t hbm_budget_bytes, int streams,
                          int max_group, fg_server **out);
fg_status fg_server_submit(fg_server *srv, const fg_request *req, uint64_t *ticket);
/* Waits up to timeout_ms (<0: forever) for the ticket; FG_ERR_TIMEOUT if
 * it has not completed. */
fg_status fg_server_wait(fg_server *srv, uint64_t ticket, int64_t timeout_ms);
/* fg_server_wait that also returns when the ticket was submitted and when
 * its work was seen complete on the GPU, in seconds of fg_server_clock, so
 * a caller that waits on tickets in any order still gets each request's
 * own completion time. */
fg_status fg_server_wait_times(fg_server *srv, uint64_t ticket, int64_t timeout_ms,
                               double *submit_s, double *done_s);
/* The server's monotonic clock in seconds. */
double fg_server_clock(void);
fg_status fg_server_stats_get(fg_server *srv, fg_server_stats *out);
fg_status fg_server_stop(fg_server *srv);

#ifdef __cplusplus
}
#endif

#endif /* FERRAY_GPU_H */
