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
 * Threads and data movement of the real-valued GEMMs (f64, f32) follow
 * ferray's driver so that the timed CPU baseline runs like ferray: a pool of
 * min(cores, 8) threads (outer.rs:142-155), the parallel switch
 * max(m, n, k) >= 256 and m >= 2 MR (outer.rs:162, 233, 531), pick_grid's
 * 1-D M-slab or 2-D M x N grid (outer.rs:343-383, 692-726) with MR / NR
 * rounded cells (outer.rs:249-250), and per cell the sequential 5-loop with
 * B packed into NR-wide strips per (NC, KC) panel and A into MR-high strips
 * per MC block (outer.rs:393-488, pack.rs pack_a / pack_b / pack_a_f32 /
 * pack_b_f32), the micro-kernel reading both packs sequentially.  Complex and
 * integer GEMMs split rows over the same pool.  No split changes a result:
 * every element's arithmetic is independent of the grid and of packing.
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

/* pick_grid / pick_grid_f32 (outer.rs:343-383, 692-726): 1-D M-slab when
 * every worker gets at least one MR strip and one worker's B pack
 * (min(KC, k) x n elements) fits the per-worker L2 budget, otherwise the
 * mw x nw factorisation of the pool (mw <= m / MR) whose cells are closest
 * to square in log scale, ties to the larger mw. */
static void pick_grid(size_t m, size_t n, size_t k, size_t workers, size_t mr,
                      size_t budget, size_t *mw_out, size_t *nw_out) {
    *mw_out = workers ? workers : 1;
    *nw_out = 1;
    if (workers <= 1 || m == 0 || n == 0) return;
    size_t kc_eff = k < FR_KC ? (k ? k : 1) : FR_KC;
    size_t mr_chunks = m / mr;
    if (mr_chunks >= workers && kc_eff * n <= budget) return;
    size_t mw_max = mr_chunks ? mr_chunks : 1;
    size_t best_m = 1, best_n = workers;
    double best = INFINITY;
    for (size_t mw = 1; mw <= mw_max && mw <= workers; mw++) {
        if (workers % mw) continue;
        size_t nw = workers / mw;
        double score = fabs(log((double)m / (double)mw) - log((double)n / (double)nw));
        if (score < best || (score == best && mw > best_m)) {
            best_m = mw; best_n = nw; best = score;
        }
    }
    *mw_out = best_m;
    *nw_out = best_n;
}

/* The grid cells of outer.rs:249-270: per-cell sizes rounded up to MR / NR
 * multiples, cells in row-major order. */
typedef struct { size_t m0, ms, n0, ns; } fr_cell;

static size_t make_cells(size_t m, size_t n, size_t mw, size_t nw, size_t mr,
                         size_t nr, fr_cell *cells) {
    size_t m_per = (m + mw - 1) / mw, n_per = (n + nw - 1) / nw;
    m_per = (m_per + mr - 1) / mr * mr;
    n_per = (n_per + nr - 1) / nr * nr;
    if (m_per < mr) m_per = mr;
    if (n_per < nr) n_per = nr;
    size_t cnt = 0;
    for (size_t i = 0; i < m; i += m_per)
        for (size_t j = 0; j < n; j += n_per) {
            fr_cell c = {i, (m - i) < m_per ? (m - i) : m_per, j, (n - j) < n_per ? (n - j) : n_per};
            cells[cnt++] = c;
        }
    return cnt;
}

/* Packed micro-kernel for a full 4x8 tile: pa = MR-interleaved A strip
 * (pa[p*4 + i]), pb = NR-interleaved B strip (pb[p*8 + j]); one
 * fused-multiply-add chain per element, then alpha and the store rule of
 * kernel_avx2.rs:167-208 (beta == 0: store, beta == 1: add, else
 * fma(C, beta, v)). */
static void ukr_f64_4x8(size_t kc, double alpha, const double *pa, const double *pb,
                        double beta, double *c, size_t ldc) {
    __m256d c00 = _mm256_setzero_pd(), c01 = _mm256_setzero_pd();
    __m256d c10 = _mm256_setzero_pd(), c11 = _mm256_setzero_pd();
    __m256d c20 = _mm256_setzero_pd(), c21 = _mm256_setzero_pd();
    __m256d c30 = _mm256_setzero_pd(), c31 = _mm256_setzero_pd();
    for (size_t p = 0; p < kc; p++) {
        _mm_prefetch((const char *)(pa + 64), _MM_HINT_T0);
        _mm_prefetch((const char *)(pb + 20), _MM_HINT_T0);
        __m256d b0 = _mm256_loadu_pd(pb), b1 = _mm256_loadu_pd(pb + 4);
        __m256d a0 = _mm256_broadcast_sd(pa);
        c00 = _mm256_fmadd_pd(a0, b0, c00); c01 = _mm256_fmadd_pd(a0, b1, c01);
        __m256d a1 = _mm256_broadcast_sd(pa + 1);
        c10 = _mm256_fmadd_pd(a1, b0, c10); c11 = _mm256_fmadd_pd(a1, b1, c11);
        __m256d a2 = _mm256_broadcast_sd(pa + 2);
        c20 = _mm256_fmadd_pd(a2, b0, c20); c21 = _mm256_fmadd_pd(a2, b1, c21);
        __m256d a3 = _mm256_broadcast_sd(pa + 3);
        c30 = _mm256_fmadd_pd(a3, b0, c30); c31 = _mm256_fmadd_pd(a3, b1, c31);
        pa += 4; pb += 8;
    }
    __m256d acc[4][2] = {{c00, c01}, {c10, c11}, {c20, c21}, {c30, c31}};
    __m256d al = _mm256_set1_pd(alpha), be = _mm256_set1_pd(beta);
    for (int i = 0; i < 4; i++)
        for (int h = 0; h < 2; h++) {
            __m256d v = acc[i][h];
            if (alpha != 1.0) v = _mm256_mul_pd(v, al);
            double *pc = c + i * ldc + 4 * h;
            if (beta == 0.0) _mm256_storeu_pd(pc, v);
            else if (beta == 1.0) _mm256_storeu_pd(pc, _mm256_add_pd(_mm256_loadu_pd(pc), v));
            else _mm256_storeu_pd(pc, _mm256_fmadd_pd(_mm256_loadu_pd(pc), be, v));
        }
}

/* Packing (pack.rs): A block (mc x kc) into MR-high strips, B panel
 * (kc x nc) into NR-wide strips, zero padded. */
#define DEFINE_PACK(SUF, T)                                                        \
static void pack_a_##SUF(size_t mc, size_t kc, const T *a, size_t lda, size_t mr,  \
                         T *out) {                                                 \
    for (size_t s = 0; s * mr < mc; s++) {                                         \
        size_t r0 = s * mr, rows = (mc - r0) < mr ? (mc - r0) : mr;                \
        T *strip = out + s * mr * kc;                                              \
        for (size_t p = 0; p < kc; p++)                                            \
            for (size_t i = 0; i < mr; i++)                                        \
                strip[p * mr + i] = i < rows ? a[(r0 + i) * lda + p] : (T)0;       \
    }                                                                              \
}                                                                                  \
static void pack_b_##SUF(size_t kc, size_t nc, const T *b, size_t ldb, size_t nr,  \
                         T *out) {                                                 \
    for (size_t s = 0; s * nr < nc; s++) {                                         \
        size_t c0 = s * nr, cols = (nc - c0) < nr ? (nc - c0) : nr;                \
        T *strip = out + s * nr * kc;                                              \
        if (cols == nr) {                                                          \
            for (size_t p = 0; p < kc; p++)                                        \
                memcpy(strip + p * nr, b + p * ldb + c0, nr * sizeof(T));          \
        } else {                                                                   \
            for (size_t p = 0; p < kc; p++)                                        \
                for (size_t j = 0; j < nr; j++)                                    \
                    strip[p * nr + j] = j < cols ? b[p * ldb + c0 + j] : (T)0;     \
        }                                                                          \
    }                                                                              \
}
DEFINE_PACK(f64, double)
DEFINE_PACK(f32, float)

/* Per-thread pack buffers (outer.rs:79-134 keeps them thread-local). */
static __thread double *tls_pa64, *tls_pb64;
static __thread float *tls_pa32, *tls_pb32;

/* gemm_seq_avx2_f64 (outer.rs:393-488) on one cell: NC panels of B, KC
 * panels with beta on the first only, MC blocks of A; full tiles on the
 * packed micro-kernel, ragged tiles on the scalar edge kernel. */
static void seq_f64(size_t m, size_t n, size_t k, double alpha, const double *a, size_t lda,
                    const double *b, size_t ldb, double beta, double *c, size_t ldc) {
    const size_t MR = 4, NR = 8;
    if (!tls_pb64) {
        tls_pb64 = (double *)aligned_alloc(64, FR_KC * FR_NC * sizeof(double));
        tls_pa64 = (double *)aligned_alloc(64, FR_MC * FR_KC * sizeof(double));
    }
    for (size_t jc = 0; jc < n; jc += FR_NC) {
        size_t nc = (n - jc) < FR_NC ? (n - jc) : FR_NC;
        for (size_t pc = 0; pc < k; pc += FR_KC) {
            size_t kc = (k - pc) < FR_KC ? (k - pc) : FR_KC;
            double eb = pc == 0 ? beta : 1.0;
            pack_b_f64(kc, nc, b + pc * ldb + jc, ldb, NR, tls_pb64);
            for (size_t ic = 0; ic < m; ic += FR_MC) {
                size_t mc = (m - ic) < FR_MC ? (m - ic) : FR_MC;
                pack_a_f64(mc, kc, a + ic * lda + pc, lda, MR, tls_pa64);
                for (size_t jr = 0; jr < nc; jr += NR)
                    for (size_t ir = 0; ir < mc; ir += MR) {
                        size_t mt = (mc - ir) < MR ? (mc - ir) : MR;
                        size_t nt = (nc - jr) < NR ? (nc - jr) : NR;
                        double *cp = c + (ic + ir) * ldc + jc + jr;
                        if (mt == MR && nt == NR)
                            ukr_f64_4x8(kc, alpha, tls_pa64 + ir * kc, tls_pb64 + jr * kc, eb, cp, ldc);
                        else
                            tile_f64_edge(mt, nt, kc, alpha, a + (ic + ir) * lda + pc, lda,
                                          b + pc * ldb + jc + jr, ldb, eb, cp, ldc);
                    }
            }
        }
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
    size_t mx = m > n ? m : n; mx = mx > k ? mx : k;
    if (!(mx >= 256 && m >= 2 * MR)) { /* outer.rs:233: sequential */
        seq_f64(m, n, k, alpha, a, k, b, n, beta, c, n);
        return 1;
    }
    size_t workers = (size_t)nthreads(), mw, nw;
    pick_grid(m, n, k, workers, MR, 128 * 1024, &mw, &nw);
    fr_cell *cells = (fr_cell *)malloc(mw * nw * 4 * sizeof(fr_cell) + sizeof(fr_cell));
    size_t cnt = make_cells(m, n, mw, nw, MR, NR, cells);
#pragma omp parallel for schedule(dynamic, 1) num_threads((int)workers)
    for (size_t q = 0; q < cnt; q++) {
        fr_cell cl = cells[q];
        seq_f64(cl.ms, cl.ns, k, alpha, a + cl.m0 * k, k, b + cl.n0, n, beta,
                c + cl.m0 * n + cl.n0, n);
    }
    free(cells);
    return 1;
}

/* ------------------------------------------------------------------ */
/* f32: 4x16 tiles                                                      */
/* ------------------------------------------------------------------ */

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

/* Packed 4x16 micro-kernel (kernel_avx2_f32.rs:56-235 reads packed strips
 * the same way): the chains and store rule of ukr_f64_4x8 in f32. */
static void ukr_f32_4x16(size_t kc, float alpha, const float *pa, const float *pb,
                         float beta, float *c, size_t ldc) {
    __m256 c00 = _mm256_setzero_ps(), c01 = _mm256_setzero_ps();
    __m256 c10 = _mm256_setzero_ps(), c11 = _mm256_setzero_ps();
    __m256 c20 = _mm256_setzero_ps(), c21 = _mm256_setzero_ps();
    __m256 c30 = _mm256_setzero_ps(), c31 = _mm256_setzero_ps();
    for (size_t p = 0; p < kc; p++) {
        _mm_prefetch((const char *)(pa + 128), _MM_HINT_T0);
        _mm_prefetch((const char *)(pb + 40), _MM_HINT_T0);
        _mm_prefetch((const char *)(pb + 48), _MM_HINT_T0);
        __m256 b0 = _mm256_loadu_ps(pb), b1 = _mm256_loadu_ps(pb + 8);
        __m256 a0 = _mm256_broadcast_ss(pa);
        c00 = _mm256_fmadd_ps(a0, b0, c00); c01 = _mm256_fmadd_ps(a0, b1, c01);
        __m256 a1 = _mm256_broadcast_ss(pa + 1);
        c10 = _mm256_fmadd_ps(a1, b0, c10); c11 = _mm256_fmadd_ps(a1, b1, c11);
        __m256 a2 = _mm256_broadcast_ss(pa + 2);
        c20 = _mm256_fmadd_ps(a2, b0, c20); c21 = _mm256_fmadd_ps(a2, b1, c21);
        __m256 a3 = _mm256_broadcast_ss(pa + 3);
        c30 = _mm256_fmadd_ps(a3, b0, c30); c31 = _mm256_fmadd_ps(a3, b1, c31);
        pa += 4; pb += 16;
    }
    __m256 acc[4][2] = {{c00, c01}, {c10, c11}, {c20, c21}, {c30, c31}};
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

/* gemm_seq_avx2_f32 (outer.rs:593-680), as seq_f64 with 4x16 tiles. */
static void seq_f32(size_t m, size_t n, size_t k, float alpha, const float *a, size_t lda,
                    const float *b, size_t ldb, float beta, float *c, size_t ldc) {
    const size_t MR = 4, NR = 16;
    if (!tls_pb32) {
        tls_pb32 = (float *)aligned_alloc(64, FR_KC * FR_NC * sizeof(float));
        tls_pa32 = (float *)aligned_alloc(64, FR_MC * FR_KC * sizeof(float));
    }
    for (size_t jc = 0; jc < n; jc += FR_NC) {
        size_t nc = (n - jc) < FR_NC ? (n - jc) : FR_NC;
        for (size_t pc = 0; pc < k; pc += FR_KC) {
            size_t kc = (k - pc) < FR_KC ? (k - pc) : FR_KC;
            float eb = pc == 0 ? beta : 1.0f;
            pack_b_f32(kc, nc, b + pc * ldb + jc, ldb, NR, tls_pb32);
            for (size_t ic = 0; ic < m; ic += FR_MC) {
                size_t mc = (m - ic) < FR_MC ? (m - ic) : FR_MC;
                pack_a_f32(mc, kc, a + ic * lda + pc, lda, MR, tls_pa32);
                for (size_t jr = 0; jr < nc; jr += NR)
                    for (size_t ir = 0; ir < mc; ir += MR) {
                        size_t mt = (mc - ir) < MR ? (mc - ir) : MR;
                        size_t nt = (nc - jr) < NR ? (nc - jr) : NR;
                        float *cp = c + (ic + ir) * ldc + jc + jr;
                        if (mt == MR && nt == NR)
                            ukr_f32_4x16(kc, alpha, tls_pa32 + ir * kc, tls_pb32 + jr * kc, eb, cp, ldc);
                        else
                            tile_f32_edge(mt, nt, kc, alpha, a + (ic + ir) * lda + pc, lda,
                                          b + pc * ldb + jc + jr, ldb, eb, cp, ldc);
                    }
            }
        }
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
    size_t mx = m > n ? m : n; mx = mx > k ? mx : k;
    if (!(mx >= 256 && m >= 2 * MR)) { /* outer.rs:531: sequential */
        seq_f32(m, n, k, alpha, a, k, b, n, beta, c, n);
        return 1;
    }
    size_t workers = (size_t)nthreads(), mw, nw;
    pick_grid(m, n, k, workers, MR, 256 * 1024, &mw, &nw);
    fr_cell *cells = (fr_cell *)malloc(mw * nw * 4 * sizeof(fr_cell) + sizeof(fr_cell));
    size_t cnt = make_cells(m, n, mw, nw, MR, NR, cells);
#pragma omp parallel for schedule(dynamic, 1) num_threads((int)workers)
    for (size_t q = 0; q < cnt; q++) {
        fr_cell cl = cells[q];
        seq_f32(cl.ms, cl.ns, k, alpha, a + cl.m0 * k, k, b + cl.n0, n, beta,
                c + cl.m0 * n + cl.n0, n);
    }
    free(cells);
    return 1;
}

/* The grid ferray picks for an f64 / f32 GEMM on `workers` threads, for the
 * tests: writes (mw, nw); returns 0 when the call would run sequentially. */
int fr_pick_grid(size_t m, size_t n, size_t k, size_t workers, int is_f32, size_t *mw,
                 size_t *nw) {
    size_t mr = 4;
    size_t mx = m > n ? m : n; mx = mx > k ? mx : k;
    pick_grid(m, n, k, workers, mr, is_f32 ? 256 * 1024 : 128 * 1024, mw, nw);
    return mx >= 256 && m >= 2 * mr;
}

/* ------------------------------------------------------------------ */
/* complex (interleaved re,im), generic over double / float             */
/* ------------------------------------------------------------------ */

#define DEFINE_COMPLEX(SUF, T, FMA, MR, NR, BUDGET)                                          \
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
    size_t mx = m > n ? m : n; mx = mx > k ? mx : k;                                \
    size_t workers = (size_t)nthreads(), mw = 1, nw = 1;                           \
    if (mx >= 256 && m >= 2 * MR)                                                   \
        pick_grid(m, n, k, workers, 4, BUDGET, &mw, &nw);                           \
    fr_cell *cells = (fr_cell *)malloc(mw * nw * 4 * sizeof(fr_cell) + sizeof(fr_cell)); \
    size_t cnt = make_cells(m, n, mw, nw, MR, NR, cells);                           \
    _Pragma("omp parallel for schedule(dynamic, 1) num_threads((int)workers)")      \
    for (size_t q = 0; q < cnt; q++) {                                              \
        fr_cell cl = cells[q];                                                      \
        const T *ac = a + 2 * cl.m0 * k, *bc = b + 2 * cl.n0;                       \
        T *cc = c + 2 * (cl.m0 * n + cl.n0);                                        \
        for (size_t jc = 0; jc < cl.ns; jc += FR_NC) {                              \
            size_t nc = (cl.ns - jc) < FR_NC ? (cl.ns - jc) : FR_NC;                \
            for (size_t pc = 0; pc < k; pc += FR_KC) {                              \
                size_t kc = (k - pc) < FR_KC ? (k - pc) : FR_KC;                    \
                T ebr = pc == 0 ? br_ : (T)1, ebi = pc == 0 ? bi_ : (T)0;           \
                for (size_t ic = 0; ic < cl.ms; ic += FR_MC) {                      \
                    size_t mc = (cl.ms - ic) < FR_MC ? (cl.ms - ic) : FR_MC;        \
                    for (size_t jr = 0; jr < nc; jr += NR)                          \
                        for (size_t irr = 0; irr < mc; irr += MR) {                 \
                            size_t i0 = ic + irr, j0 = jc + jr;                     \
                            size_t mt = (mc - irr) < MR ? (mc - irr) : MR;          \
                            size_t nt = (nc - jr) < NR ? (nc - jr) : NR;            \
                            const T *ap = ac + 2 * (i0 * k + pc);                   \
                            const T *bp = bc + 2 * (pc * n + j0);                   \
                            T *cp = cc + 2 * (i0 * n + j0);                         \
                            if (mt == MR && nt == NR)                               \
                                ctile_full_##SUF(kc, ar_, ai_, ap, k, bp, n, ebr, ebi, cp, n); \
                            else                                                    \
                                ctile_edge_##SUF(mt, nt, kc, ar_, ai_, ap, k, bp, n, ebr, ebi, cp, n); \
                        }                                                           \
                }                                                                   \
            }                                                                       \
        }                                                                           \
    }                                                                               \
    free(cells);                                                                    \
    return 1;                                                                       \
}

DEFINE_COMPLEX(c64, double, fma, 4, 2, 128 * 1024)
DEFINE_COMPLEX(c32, float, fmaf, 4, 4, 256 * 1024)

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

DEFINE_INT_GEMM(fr_gemm_i8_signed_rows, int8_t, int8_t)
DEFINE_INT_GEMM(fr_gemm_i16, int16_t, int16_t)
DEFINE_INT_GEMM(fr_gemm_i8_vnni, uint8_t, int8_t)

/* i8 x i8 -> i32 as ferray runs it (gemm_avx2_i8s, outer.rs:2682-2900):
 * the pick_grid cells, KC panels, A packed into MR-high strips widened to
 * int16 pairs (pack.rs pack_a_i8s), B packed into NR-wide strips of (k, k+1)
 * byte pairs (pack_kc_i8s), and the 4x8 vpmaddwd micro-kernel
 * (kernel_avx2_i8s.rs:63-129).  Sums are exact mod 2^32, so every order
 * gives the same bits as fr_gemm_i8_signed_rows. */
static void ukr_i8s_4x8(size_t kp, const int16_t *pa, const int8_t *pb, int32_t *c, size_t ldc,
                        int accumulate) {
    __m256i acc0 = _mm256_setzero_si256(), acc1 = _mm256_setzero_si256();
    __m256i acc2 = _mm256_setzero_si256(), acc3 = _mm256_setzero_si256();
    for (size_t q = 0; q < kp; q++) {
        _mm_prefetch((const char *)pa + 512, _MM_HINT_T0);
        _mm_prefetch((const char *)pb + 512, _MM_HINT_T0);
        __m256i bv = _mm256_cvtepi8_epi16(_mm_loadu_si128((const __m128i *)pb));
        int32_t w;
        memcpy(&w, pa, 4); acc0 = _mm256_add_epi32(acc0, _mm256_madd_epi16(_mm256_set1_epi32(w), bv));
        memcpy(&w, pa + 2, 4); acc1 = _mm256_add_epi32(acc1, _mm256_madd_epi16(_mm256_set1_epi32(w), bv));
        memcpy(&w, pa + 4, 4); acc2 = _mm256_add_epi32(acc2, _mm256_madd_epi16(_mm256_set1_epi32(w), bv));
        memcpy(&w, pa + 6, 4); acc3 = _mm256_add_epi32(acc3, _mm256_madd_epi16(_mm256_set1_epi32(w), bv));
        pa += 8; pb += 16;
    }
    __m256i acc[4] = {acc0, acc1, acc2, acc3};
    for (int i = 0; i < 4; i++) {
        __m256i *pc = (__m256i *)(c + i * ldc);
        __m256i v = acc[i];
        if (accumulate) v = _mm256_add_epi32(v, _mm256_loadu_si256(pc));
        _mm256_storeu_si256(pc, v);
    }
}

static __thread int16_t *tls_pa_i8;
static __thread int8_t *tls_pb_i8;

static void seq_i8s(size_t m, size_t n, size_t k, const int8_t *a, size_t lda, const int8_t *b,
                    size_t ldb, int32_t *c, size_t ldc, int accumulate) {
    const size_t MR = 4, NR = 8;
    if (!tls_pb_i8) {
        tls_pb_i8 = (int8_t *)aligned_alloc(64, (FR_KC + 2) * FR_NC);
        tls_pa_i8 = (int16_t *)aligned_alloc(64, FR_MC * (FR_KC + 2) * sizeof(int16_t));
    }
    for (size_t jc = 0; jc < n; jc += FR_NC) {
        size_t nc = (n - jc) < FR_NC ? (n - jc) : FR_NC;
        size_t nstrips = (nc + NR - 1) / NR;
        for (size_t pc = 0; pc < k; pc += FR_KC) {
            size_t kc = (k - pc) < FR_KC ? (k - pc) : FR_KC;
            size_t kp = (kc + 1) / 2;  /* k pairs, the odd tail zero padded */
            int acc = pc == 0 ? accumulate : 1;
            for (size_t s = 0; s < nstrips; s++) {
                int8_t *strip = tls_pb_i8 + s * kp * 16;
                for (size_t q = 0; q < kp; q++)
                    for (size_t j = 0; j < NR; j++) {
                        size_t col = jc + s * NR + j, k0 = pc + 2 * q;
                        int live = col < jc + nc;
                        strip[q * 16 + 2 * j] = live ? b[k0 * ldb + col] : 0;
                        strip[q * 16 + 2 * j + 1] = (live && 2 * q + 1 < kc) ? b[(k0 + 1) * ldb + col] : 0;
                    }
            }
            for (size_t ic = 0; ic < m; ic += FR_MC) {
                size_t mc = (m - ic) < FR_MC ? (m - ic) : FR_MC;
                for (size_t r = 0; r * MR < mc; r++) {
                    int16_t *strip = tls_pa_i8 + r * kp * 8;
                    for (size_t q = 0; q < kp; q++)
                        for (size_t i = 0; i < MR; i++) {
                            size_t row = ic + r * MR + i, k0 = pc + 2 * q;
                            int live = row < ic + mc;
                            strip[q * 8 + 2 * i] = live ? a[row * lda + k0] : 0;
                            strip[q * 8 + 2 * i + 1] = (live && 2 * q + 1 < kc) ? a[row * lda + k0 + 1] : 0;
                        }
                }
                for (size_t jr = 0; jr < nc; jr += NR)
                    for (size_t ir = 0; ir < mc; ir += MR) {
                        size_t mt = (mc - ir) < MR ? (mc - ir) : MR;
                        size_t nt = (nc - jr) < NR ? (nc - jr) : NR;
                        int32_t *cp = c + (ic + ir) * ldc + jc + jr;
                        const int16_t *pa = tls_pa_i8 + (ir / MR) * kp * 8;
                        const int8_t *pb = tls_pb_i8 + (jr / NR) * kp * 16;
                        if (mt == MR && nt == NR) {
                            ukr_i8s_4x8(kp, pa, pb, cp, ldc, acc);
                        } else {  /* ragged edge: exact scalar sums from the packs */
                            for (size_t i = 0; i < mt; i++)
                                for (size_t j = 0; j < nt; j++) {
                                    uint32_t v = 0;
                                    for (size_t q = 0; q < kp; q++)
                                        v += (uint32_t)((int32_t)pa[q * 8 + 2 * i] * pb[q * 16 + 2 * j] +
                                                        (int32_t)pa[q * 8 + 2 * i + 1] * pb[q * 16 + 2 * j + 1]);
                                    if (acc) v += (uint32_t)cp[i * ldc + j];
                                    cp[i * ldc + j] = (int32_t)v;
                                }
                        }
                    }
            }
        }
    }
}

int fr_gemm_i8_signed(size_t m, size_t n, size_t k, const int8_t *a, const int8_t *b,
                      int32_t *c, int accumulate) {
    if (m == 0 || n == 0) return 1;
    if (k == 0) {
        if (!accumulate) memset(c, 0, m * n * sizeof(int32_t));
        return 1;
    }
    const size_t MR = 4, NR = 8;
    size_t mx = m > n ? m : n; mx = mx > k ? mx : k;
    if (!(mx >= 256 && m >= 2 * MR)) {
        seq_i8s(m, n, k, a, k, b, n, c, n, accumulate);
        return 1;
    }
    size_t workers = (size_t)nthreads(), mw, nw;
    pick_grid(m, n, k, workers, MR, 128 * 1024, &mw, &nw);
    fr_cell *cells = (fr_cell *)malloc(mw * nw * 4 * sizeof(fr_cell) + sizeof(fr_cell));
    size_t cnt = make_cells(m, n, mw, nw, MR, NR, cells);
#pragma omp parallel for schedule(dynamic, 1) num_threads((int)workers)
    for (size_t q = 0; q < cnt; q++) {
        fr_cell cl = cells[q];
        seq_i8s(cl.ms, cl.ns, k, a + cl.m0 * k, k, b + cl.n0, n, c + cl.m0 * n + cl.n0, n, accumulate);
    }
    free(cells);
    return 1;
}

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
