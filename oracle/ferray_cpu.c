/*
 * ferray_cpu.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * A C restatement of ferray-linalg's CPU GEMM for every dtype on the matmul
 * path.  It exists to (1) check the CUDA backend bit-for-bit on the integer
 * paths, (2) show how far ferray's own float results sit from the
 * double-double oracle (dd_oracle.c), and (3) serve as the timed CPU
 * baseline.  Nothing in the product library links or calls this file.
 *
 * What is restated, with the reference file it follows (paths are inside
 * the ferray workspace):
 *
 *  - Blocking MC=64, KC=256, NC=512 (ferray-linalg/src/gemm/outer.rs:66-68)
 *    and beta applied on the first KC panel only, later panels adding into C
 *    (outer.rs:415-421, 483).  The K loop therefore restarts from zero every
 *    256 elements and the panel partial sums are added to C in panel order.
 *  - The default (no cargo feature) x86 AVX2 register tiles:
 *      f64 4x8   (gemm/kernel_avx2.rs:53-193, edge :251-290)
 *      f32 4x16  (gemm/kernel_avx2_f32.rs:56-235)
 *      c64 4x2   (gemm/kernel_avx2_complex_f64.rs:79-186, edge :262-312)
 *      c32 4x4   (gemm/kernel_avx2_complex_f32.rs:63-170)
 *    Every C element is one fused-multiply-add chain per panel, which is what
 *    each SIMD lane of those kernels computes, so a scalar fma() per element
 *    reproduces the lane results bit for bit.  Elements in a full MRxNR tile
 *    use the kernel's store (beta != 0,1 -> fma(C, beta, v)); elements of the
 *    ragged edge use the scalar edge kernel's store (beta*C + v, unfused).
 *    Tiles are full exactly for i < floor(m/MR)*MR and j < floor(n/NR)*NR
 *    because every grid chunk and block size is an MR/NR multiple
 *    (outer.rs:233-240, 343-383).
 *  - Complex tiles keep four real accumulators per element (Re*Re, Re*Im,
 *    Im*Im, Im*Re) and combine them with add/sub after the panel, exactly
 *    the vaddsubpd scheme (kernel_avx2_complex_f64.rs:103-158); alpha and
 *    beta use the same broadcast/swap/addsub arithmetic (:160-226).  Edge
 *    tiles use the unfused scalar complex product (:262-312).
 *  - Integers: i8xi8 (kernel_avx2_i8s.rs:63-129) and i16xi16
 *    (kernel_avx2_i16.rs:52-117) are exact sums mod 2^32.  u8xi8 has two
 *    variants: the default AVX2 vpmaddubsw chain, which saturates each
 *    adjacent (k, k+1) pair sum to int16 inside full 4x8 tiles
 *    (kernel_avx2_i8.rs:61-136) while edge tiles are exact (:176-215), and
 *    the avxvnni / avx512 VNNI kernels, which are exact
 *    (kernel_avx512_vnni_i8.rs:49).
 *  - quantized_matmul's zero-point/scale epilogue (gemm/mod.rs:484-575).
 *  - matmul_raw's dispatch (products/mod.rs:462-577): max_dim <= 8 takes the
 *    naive ikj loop with separately rounded multiply and add; max_dim >= 256
 *    takes gemm_f64/gemm_f32.  The 9..255 range goes to faer 0.24 in the
 *    reference; faer is not vendored, so that range is NOT bit-pinned and
 *    this file routes it through the same blocked kernel.
 *
 * Threads: rows are split over up to min(cores, 8) OpenMP threads, the size
 * of ferray's GEMM pool (outer.rs:142-155).  The split never changes a
 * result because every element's arithmetic is independent of the grid.
 */
#include <immintrin.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>

#define FR_MC 64
#define FR_KC 256
#define FR_NC 512

static int fr_threads = 0;

void fr_set_threads(int n) { fr_threads = n; }

static int nthreads(void) {
    if (fr_threads > 0) return fr_threads;
    int n = omp_get_num_procs();
    return n < 8 ? n : 8;
}

/* ------------------------------------------------------------------ */
/* f64: 4x8 tiles                                                       */
/* ------------------------------------------------------------------ */

/* One full 4x8 tile over one KC panel: fused chains, then alpha and the
 * store rule of kernel_avx2.rs:167-208. */
static void tile_f64_full(size_t kc, double alpha, const double *a, size_t lda,
                          const double *b, size_t ldb, double beta, double *c,
                          size_t ldc) {
    __m256d acc[4][2];
    for (int i = 0; i < 4; i++) acc[i][0] = acc[i][1] = _mm256_setzero_pd();
    for (size_t p = 0; p < kc; p++) {
        __m256d b0 = _mm256_loadu_pd(b + p * ldb);
        __m256d b1 = _mm256_loadu_pd(b + p * ldb + 4);
        for (int i = 0; i < 4; i++) {
            __m256d av = _mm256_broadcast_sd(a + i * lda + p);
            acc[i][0] = _mm256_fmadd_pd(av, b0, acc[i][0]);
            acc[i][1] = _mm256_fmadd_pd(av, b1, acc[i][1]);
        }
    }
    __m256d al = _mm256_set1_pd(alpha), be = _mm256_set1_pd(beta);
    for (int i = 0; i < 4; i++) {
        for (int h = 0; h < 2; h++) {
            __m256d v = acc[i][h];
            if (alpha != 1.0) v = _mm256_mul_pd(v, al);
            double *pc = c + i * ldc + 4 * h;
            if (beta == 0.0) {
                _mm256_storeu_pd(pc, v);
            } else if (beta == 1.0) {
                _mm256_storeu_pd(pc, _mm256_add_pd(_mm256_loadu_pd(pc), v));
            } else {
                _mm256_storeu_pd(pc, _mm256_fmadd_pd(_mm256_loadu_pd(pc), be, v));
            }
        }
    }
}

static void tile_f64_edge(size_t mt, size_t nt, size_t kc, double alpha,
                          const double *a, size_t lda, const double *b,
                          size_t ldb, double beta, double *c, size_t ldc) {
    double t[4][8] = {{0}};
    for (size_t p = 0; p < kc; p++)
        for (size_t i = 0; i < mt; i++) {
            double ai = a[i * lda + p];
            for (size_t j = 0; j < nt; j++) t[i][j] = fma(ai, b[p * ldb + j], t[i][j]);
        }
    for (size_t i = 0; i < mt; i++)
        for (size_t j = 0; j < nt; j++) {
            double v = alpha * t[i][j];
            double *pc = c + i * ldc + j;
            if (beta == 0.0) *pc = v;
            else if (beta == 1.0) *pc += v;
            else *pc = beta * *pc + v;
        }
}

int fr_gemm_f64(size_t m, size_t n, size_t k, double alpha, const double *a,
                const double *b, double beta, double *c) {
    if (m == 0 || n == 0) return 1;
    if (k == 0) { /* outer.rs:213-229 */
        for (size_t i = 0; i < m * n; i++) {
            if (beta == 0.0) c[i] = 0.0;
            else if (beta != 1.0) c[i] *= beta;
        }
        return 1;
    }
    const size_t MR = 4, NR = 8;
    size_t mfull = m / MR * MR, nfull = n / NR * NR;
    size_t nblk = (m + FR_MC - 1) / FR_MC;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads())
    for (size_t blk = 0; blk < nblk; blk++) {
        size_t ic = blk * FR_MC, mc = (m - ic) < FR_MC ? (m - ic) : FR_MC;
        for (size_t jc = 0; jc < n; jc += FR_NC) {
            size_t nc = (n - jc) < FR_NC ? (n - jc) : FR_NC;
            for (size_t pc = 0; pc < k; pc += FR_KC) {
                size_t kc = (k - pc) < FR_KC ? (k - pc) : FR_KC;
                double eb = pc == 0 ? beta : 1.0;
                for (size_t jr = 0; jr < nc; jr += NR)
                    for (size_t ir = 0; ir < mc; ir += MR) {
                        size_t i0 = ic + ir, j0 = jc + jr;
                        size_t mt = (m - i0) < MR ? (m - i0) : MR;
                        size_t nt = (jc + nc - j0) < NR ? (jc + nc - j0) : NR;
                        const double *ap = a + i0 * k + pc;
                        const double *bp = b + pc * n + j0;
                        double *cp = c + i0 * n + j0;
                        if (i0 + MR <= mfull && j0 + NR <= nfull && mt == MR && nt == NR)
                            tile_f64_full(kc, alpha, ap, k, bp, n, eb, cp, n);
                        else
                            tile_f64_edge(mt, nt, kc, alpha, ap, k, bp, n, eb, cp, n);
                    }
            }
        }
    }
    return 1;
}

/* ------------------------------------------------------------------ */
/* f32: 4x16 tiles                                                      */
/* ------------------------------------------------------------------ */

static void tile_f32_full(size_t kc, float alpha, const float *a, size_t lda,
                          const float *b, size_t ldb, float beta, float *c,
                          size_t ldc) {
    __m256 acc[4][2];
    for (int i = 0; i < 4; i++) acc[i][0] = acc[i][1] = _mm256_setzero_ps();
    for (size_t p = 0; p < kc; p++) {
        __m256 b0 = _mm256_loadu_ps(b + p * ldb);
        __m256 b1 = _mm256_loadu_ps(b + p * ldb + 8);
        for (int i = 0; i < 4; i++) {
            __m256 av = _mm256_broadcast_ss(a + i * lda + p);
            acc[i][0] = _mm256_fmadd_ps(av, b0, acc[i][0]);
            acc[i][1] = _mm256_fmadd_ps(av, b1, acc[i][1]);
        }
    }
    __m256 al = _mm256_set1_ps(alpha), be = _mm256_set1_ps(beta);
    for (int i = 0; i < 4; i++)
        for (int h = 0; h < 2; h++) {
            __m256 v = acc[i][h];
            if (alpha != 1.0f) v = _mm256_mul_ps(v, al);
            float *pc = c + i * ldc + 8 * h;
            if (beta == 0.0f) _mm256_storeu_ps(pc, v);
            else if (beta == 1.0f) _mm256_storeu_ps(pc, _mm256_add_ps(_mm256_loadu_ps(pc), v));
            else _mm256_storeu_ps(pc, _mm256_fmadd_ps(_mm256_loadu_ps(pc), be, v));
        }
}

static void tile_f32_edge(size_t mt, size_t nt, size_t kc, float alpha,
                          const float *a, size_t lda, const float *b,
                          size_t ldb, float beta, float *c, size_t ldc) {
    float t[4][16] = {{0}};
    for (size_t p = 0; p < kc; p++)
        for (size_t i = 0; i < mt; i++) {
            float ai = a[i * lda + p];
            for (size_t j = 0; j < nt; j++) t[i][j] = fmaf(ai, b[p * ldb + j], t[i][j]);
        }
    for (size_t i = 0; i < mt; i++)
        for (size_t j = 0; j < nt; j++) {
            float v = alpha * t[i][j];
            float *pc = c + i * ldc + j;
            if (beta == 0.0f) *pc = v;
            else if (beta == 1.0f) *pc += v;
            else *pc = beta * *pc + v;
        }
}

int fr_gemm_f32(size_t m, size_t n, size_t k, float alpha, const float *a,
                const float *b, float beta, float *c) {
    if (m == 0 || n == 0) return 1;
    if (k == 0) {
        for (size_t i = 0; i < m * n; i++) {
            if (beta == 0.0f) c[i] = 0.0f;
            else if (beta != 1.0f) c[i] *= beta;
        }
        return 1;
    }
    const size_t MR = 4, NR = 16;
    size_t mfull = m / MR * MR, nfull = n / NR * NR;
    size_t nblk = (m + FR_MC - 1) / FR_MC;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads())
    for (size_t blk = 0; blk < nblk; blk++) {
        size_t ic = blk * FR_MC, mc = (m - ic) < FR_MC ? (m - ic) : FR_MC;
        for (size_t jc = 0; jc < n; jc += FR_NC) {
            size_t nc = (n - jc) < FR_NC ? (n - jc) : FR_NC;
            for (size_t pc = 0; pc < k; pc += FR_KC) {
                size_t kc = (k - pc) < FR_KC ? (k - pc) : FR_KC;
                float eb = pc == 0 ? beta : 1.0f;
                for (size_t jr = 0; jr < nc; jr += NR)
                    for (size_t ir = 0; ir < mc; ir += MR) {
                        size_t i0 = ic + ir, j0 = jc + jr;
                        size_t mt = (m - i0) < MR ? (m - i0) : MR;
                        size_t nt = (jc + nc - j0) < NR ? (jc + nc - j0) : NR;
                        const float *ap = a + i0 * k + pc;
                        const float *bp = b + pc * n + j0;
                        float *cp = c + i0 * n + j0;
                        if (i0 + MR <= mfull && j0 + NR <= nfull && mt == MR && nt == NR)
                            tile_f32_full(kc, alpha, ap, k, bp, n, eb, cp, n);
                        else
                            tile_f32_edge(mt, nt, kc, alpha, ap, k, bp, n, eb, cp, n);
                    }
            }
        }
    }
    return 1;
}

/* ------------------------------------------------------------------ */
/* complex (interleaved re,im), generic over double / float             */
/* ------------------------------------------------------------------ */

#define DEFINE_COMPLEX(SUF, T, FMA, MR, NR)                                          \
static void ctile_full_##SUF(size_t kc, T ar_, T ai_, const T *a, size_t lda,      \
                             const T *b, size_t ldb, T br_, T bi_, T *c,            \
                             size_t ldc) {                                          \
    /* four chains per element: re*re, re*im, im*im, im*re */                      \
    T rr[MR][NR] = {{0}}, ri[MR][NR] = {{0}}, ii[MR][NR] = {{0}}, ir[MR][NR] = {{0}}; \
    for (size_t p = 0; p < kc; p++)                                                 \
        for (int i = 0; i < MR; i++) {                                              \
            T xr = a[2 * (i * lda + p)], xi = a[2 * (i * lda + p) + 1];             \
            for (int j = 0; j < NR; j++) {                                          \
                T yr = b[2 * (p * ldb + j)], yi = b[2 * (p * ldb + j) + 1];         \
                rr[i][j] = FMA(xr, yr, rr[i][j]);                                   \
                ri[i][j] = FMA(xr, yi, ri[i][j]);                                   \
                ii[i][j] = FMA(xi, yi, ii[i][j]);                                   \
                ir[i][j] = FMA(xi, yr, ir[i][j]);                                   \
            }                                                                       \
        }                                                                           \
    for (int i = 0; i < MR; i++)                                                    \
        for (int j = 0; j < NR; j++) {                                              \
            T vr = rr[i][j] - ii[i][j], vi = ri[i][j] + ir[i][j];                  \
            if (!(ar_ == (T)1 && ai_ == (T)0)) {                                    \
                T tr = ar_ * vr, ti = ar_ * vi; /* alpha_re * c */                  \
                T sr = ai_ * vi, si = ai_ * vr; /* alpha_im * swap(c) */            \
                vr = tr - sr; vi = ti + si;                                         \
            }                                                                       \
            T *pc = c + 2 * (i * ldc + j);                                          \
            if (br_ == (T)0 && bi_ == (T)0) { pc[0] = vr; pc[1] = vi; }             \
            else if (br_ == (T)1 && bi_ == (T)0) { pc[0] = pc[0] + vr; pc[1] = pc[1] + vi; } \
            else {                                                                  \
                T cr = pc[0], ci = pc[1];                                           \
                T tr = br_ * cr, ti = br_ * ci, sr = bi_ * ci, si = bi_ * cr;       \
                T scr = tr - sr, sci = ti + si;                                     \
                pc[0] = scr + vr; pc[1] = sci + vi;                                 \
            }                                                                       \
        }                                                                           \
}                                                                                   \
static void ctile_edge_##SUF(size_t mt, size_t nt, size_t kc, T ar_, T ai_,        \
                             const T *a, size_t lda, const T *b, size_t ldb, T br_, \
                             T bi_, T *c, size_t ldc) {                             \
    T tr[MR][NR] = {{0}}, ti[MR][NR] = {{0}};                                       \
    for (size_t p = 0; p < kc; p++)                                                 \
        for (size_t i = 0; i < mt; i++) {                                           \
            T xr = a[2 * (i * lda + p)], xi = a[2 * (i * lda + p) + 1];             \
            for (size_t j = 0; j < nt; j++) {                                       \
                T yr = b[2 * (p * ldb + j)], yi = b[2 * (p * ldb + j) + 1];         \
                T p1 = xr * yr, p2 = xi * yi, p3 = xr * yi, p4 = xi * yr;           \
                tr[i][j] += p1 - p2;                                                \
                ti[i][j] += p3 + p4;                                                \
            }                                                                       \
        }                                                                           \
    for (size_t i = 0; i < mt; i++)                                                 \
        for (size_t j = 0; j < nt; j++) {                                           \
            T u1 = ar_ * tr[i][j], u2 = ai_ * ti[i][j];                             \
            T xr = u1 - u2;                                                         \
            T u3 = ar_ * ti[i][j], u4 = ai_ * tr[i][j];                             \
            T xi = u3 + u4;                                                         \
            T *pc = c + 2 * (i * ldc + j);                                          \
            if (br_ == (T)0 && bi_ == (T)0) { pc[0] = xr; pc[1] = xi; }             \
            else {                                                                  \
                T cr = pc[0], ci = pc[1];                                           \
                T w1 = br_ * cr, w2 = bi_ * ci, w3 = br_ * ci, w4 = bi_ * cr;       \
                pc[0] = (w1 - w2) + xr;                                             \
                pc[1] = (w3 + w4) + xi;                                             \
            }                                                                       \
        }                                                                           \
}                                                                                   \
int fr_gemm_##SUF(size_t m, size_t n, size_t k, T ar_, T ai_, const T *a,          \
                  const T *b, T br_, T bi_, T *c) {                                 \
    if (m == 0 || n == 0) return 1;                                                 \
    if (k == 0) {                                                                   \
        for (size_t e = 0; e < m * n; e++) {                                        \
            T cr = c[2 * e], ci = c[2 * e + 1];                                     \
            c[2 * e] = br_ * cr - bi_ * ci;                                         \
            c[2 * e + 1] = br_ * ci + bi_ * cr;                                     \
        }                                                                           \
        return 1;                                                                   \
    }                                                                               \
    size_t mfull = m / MR * MR, nfull = n / NR * NR;                                \
    size_t nblk = (m + FR_MC - 1) / FR_MC;                                          \
    _Pragma("omp parallel for schedule(dynamic, 1) num_threads(nthreads())")        \
    for (size_t blk = 0; blk < nblk; blk++) {                                       \
        size_t ic = blk * FR_MC, mc = (m - ic) < FR_MC ? (m - ic) : FR_MC;          \
        for (size_t jc = 0; jc < n; jc += FR_NC) {                                  \
            size_t nc = (n - jc) < FR_NC ? (n - jc) : FR_NC;                        \
            for (size_t pc = 0; pc < k; pc += FR_KC) {                              \
                size_t kc = (k - pc) < FR_KC ? (k - pc) : FR_KC;                    \
                T ebr = pc == 0 ? br_ : (T)1, ebi = pc == 0 ? bi_ : (T)0;           \
                for (size_t jr = 0; jr < nc; jr += NR)                              \
                    for (size_t irr = 0; irr < mc; irr += MR) {                     \
                        size_t i0 = ic + irr, j0 = jc + jr;                         \
                        size_t mt = (m - i0) < MR ? (m - i0) : MR;                  \
                        size_t nt = (jc + nc - j0) < NR ? (jc + nc - j0) : NR;      \
                        const T *ap = a + 2 * (i0 * k + pc);                        \
                        const T *bp = b + 2 * (pc * n + j0);                        \
                        T *cp = c + 2 * (i0 * n + j0);                              \
                        if (i0 + MR <= mfull && j0 + NR <= nfull && mt == MR && nt == NR) \
                            ctile_full_##SUF(kc, ar_, ai_, ap, k, bp, n, ebr, ebi, cp, n); \
                        else                                                        \
                            ctile_edge_##SUF(mt, nt, kc, ar_, ai_, ap, k, bp, n, ebr, ebi, cp, n); \
                    }                                                               \
            }                                                                       \
        }                                                                           \
    }                                                                               \
    return 1;                                                                       \
}

DEFINE_COMPLEX(c64, double, fma, 4, 2)
DEFINE_COMPLEX(c32, float, fmaf, 4, 4)

/* ------------------------------------------------------------------ */
/* integer GEMMs                                                        */
/* ------------------------------------------------------------------ */

/* i8 x i8 -> i32 and i16 x i16 -> i32: exact sums mod 2^32
 * (kernel_avx2_i8s.rs:63-129, kernel_avx2_i16.rs:52-117). */
#define DEFINE_INT_GEMM(NAME, TA, TB)                                               \
int NAME(size_t m, size_t n, size_t k, const TA *a, const TB *b, int32_t *c,       \
         int accumulate) {                                                          \
    if (m == 0 || n == 0) return 1;                                                 \
    _Pragma("omp parallel for schedule(dynamic, 4) num_threads(nthreads())")        \
    for (size_t i = 0; i < m; i++) {                                                \
        uint32_t *row = (uint32_t *)malloc(n * sizeof(uint32_t));                   \
        for (size_t j = 0; j < n; j++) row[j] = 0;                                  \
        for (size_t p = 0; p < k; p++) {                                            \
            int32_t av = (int32_t)a[i * k + p];                                     \
            const TB *bp = b + p * n;                                               \
            for (size_t j = 0; j < n; j++)                                          \
                row[j] += (uint32_t)(av * (int32_t)bp[j]);                          \
        }                                                                           \
        for (size_t j = 0; j < n; j++) {                                            \
            uint32_t v = row[j];                                                    \
            if (accumulate) v += (uint32_t)c[i * n + j];                            \
            c[i * n + j] = (int32_t)v;                                              \
        }                                                                           \
        free(row);                                                                  \
    }                                                                               \
    return 1;                                                                       \
}

DEFINE_INT_GEMM(fr_gemm_i8_signed, int8_t, int8_t)
DEFINE_INT_GEMM(fr_gemm_i16, int16_t, int16_t)
DEFINE_INT_GEMM(fr_gemm_i8_vnni, uint8_t, int8_t)

static inline int32_t sat16(int32_t v) {
    return v > 32767 ? 32767 : (v < -32768 ? -32768 : v);
}

/* u8 x i8 -> i32, default AVX2 build: vpmaddubsw adds the two products of
 * each K pair (k, k+1) and saturates to int16 before widening
 * (kernel_avx2_i8.rs:97-117).  Pairs start at even k because every KC
 * panel starts at a multiple of 256 and the K tail is zero padded
 * (pack.rs pack_kc_i8).  Elements outside full 4x8 tiles take the exact
 * scalar edge kernel (kernel_avx2_i8.rs:176-215). */
int fr_gemm_i8_avx2(size_t m, size_t n, size_t k, const uint8_t *a,
                    const int8_t *b, int32_t *c, int accumulate) {
    if (m == 0 || n == 0) return 1;
    size_t mfull = m / 4 * 4, nfull = n / 8 * 8;
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads())
    for (size_t i = 0; i < m; i++) {
        for (size_t j = 0; j < n; j++) {
            int full = i < mfull && j < nfull;
            uint32_t acc = 0;
            for (size_t p = 0; p < k; p += 2) {
                int32_t s = (int32_t)a[i * k + p] * (int32_t)b[p * n + j];
                if (p + 1 < k) s += (int32_t)a[i * k + p + 1] * (int32_t)b[(p + 1) * n + j];
                acc += (uint32_t)(full ? sat16(s) : s);
            }
            if (accumulate) acc += (uint32_t)c[i * n + j];
            c[i * n + j] = (int32_t)acc;
        }
    }
    return 1;
}

/* quantized_matmul (gemm/mod.rs:484-575): raw = sum a*b (through gemm_i8),
 * then raw - a_zp*colsum(B) - b_zp*rowsum(A) + k*a_zp*b_zp in wrapping
 * i32, then scale_a*scale_b * (float)corrected, added to C when
 * accumulate.  `vnni` selects the exact u8xi8 variant for `raw`. */
int fr_quantized_matmul(size_t m, size_t n, size_t k, const uint8_t *a,
                        uint8_t a_zp, float scale_a, const int8_t *b,
                        int8_t b_zp, float scale_b, float *c, int accumulate,
                        int vnni) {
    if (m == 0 || n == 0) return 1;
    int32_t *raw = (int32_t *)calloc(m * n, sizeof(int32_t));
    if (vnni) fr_gemm_i8_vnni(m, n, k, a, b, raw, 0);
    else fr_gemm_i8_avx2(m, n, k, a, b, raw, 0);
    if (k == 0) {
        if (!accumulate) for (size_t e = 0; e < m * n; e++) c[e] = 0.0f;
        free(raw);
        return 1;
    }
    uint32_t *rs = (uint32_t *)calloc(m, sizeof(uint32_t));
    uint32_t *cs = (uint32_t *)calloc(n, sizeof(uint32_t));
    for (size_t i = 0; i < m; i++)
        for (size_t p = 0; p < k; p++) rs[i] += (uint32_t)(int32_t)a[i * k + p];
    for (size_t p = 0; p < k; p++)
        for (size_t j = 0; j < n; j++) cs[j] += (uint32_t)(int32_t)b[p * n + j];
    uint32_t azp = (uint32_t)(int32_t)a_zp, bzp = (uint32_t)(int32_t)b_zp;
    uint32_t kab = (uint32_t)k * azp * bzp;
    float scale = scale_a * scale_b;
    for (size_t i = 0; i < m; i++)
        for (size_t j = 0; j < n; j++) {
            uint32_t corr = (uint32_t)raw[i * n + j] - azp * cs[j] - bzp * rs[i] + kab;
            float out = scale * (float)(int32_t)corr;
            if (accumulate) c[i * n + j] += out;
            else c[i * n + j] = out;
        }
    free(raw); free(rs); free(cs);
    return 1;
}

/* ------------------------------------------------------------------ */
/* matmul_raw dispatch (products/mod.rs:462-577)                        */
/* ------------------------------------------------------------------ */

void fr_matmul_raw_f64(const double *a, const double *b, size_t m, size_t k,
                       size_t n, double *out) {
    memset(out, 0, m * n * sizeof(double));
    if (m == 0 || n == 0 || k == 0) return;
    size_t md = m > n ? m : n; md = md > k ? md : k;
    if (md <= 8) {
        for (size_t i = 0; i < m; i++)
            for (size_t p = 0; p < k; p++) {
                double x = a[i * k + p];
                for (size_t j = 0; j < n; j++) {
                    volatile double prod = x * b[p * n + j]; /* no contraction */
                    out[i * n + j] += prod;
                }
            }
        return;
    }
    fr_gemm_f64(m, n, k, 1.0, a, b, 0.0, out);
}

void fr_matmul_raw_f32(const float *a, const float *b, size_t m, size_t k,
                       size_t n, float *out) {
    memset(out, 0, m * n * sizeof(float));
    if (m == 0 || n == 0 || k == 0) return;
    size_t md = m > n ? m : n; md = md > k ? md : k;
    if (md <= 8) {
        for (size_t i = 0; i < m; i++)
            for (size_t p = 0; p < k; p++) {
                float x = a[i * k + p];
                for (size_t j = 0; j < n; j++) {
                    volatile float prod = x * b[p * n + j];
                    out[i * n + j] += prod;
                }
            }
        return;
    }
    fr_gemm_f32(m, n, k, 1.0f, a, b, 0.0f, out);
}
