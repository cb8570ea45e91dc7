/*
 * dd_oracle.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * Double-double reference GEMM used to judge every floating-point result of
 * the CUDA backend and of ferray's own CPU GEMM (ferray_cpu.c).  Each C
 * element is accumulated as an unevaluated sum hi+lo of two doubles with the
 * error-free transformations of Dekker (TwoProduct, here through fma) and
 * Knuth (TwoSum); the relative error of a dot product is then about
 * 2^-104 * cond, far below any FP64 kernel error this is used to measure.
 *
 * Entry points take real (f64 / f32) or interleaved complex (c128 / c64)
 * operands in row-major order and either produce the full C (small sizes)
 * or only the elements of a caller-chosen set of rows x columns (large
 * sizes).  dd_normwise_* return the normwise error
 *     ||C - C_ref||_F / (||A||_F * ||B||_F)
 * where the Frobenius norm of the difference is taken over the sampled
 * elements and scaled up by (m*n)/(rows*cols) so sampled and full figures
 * are comparable.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <omp.h>

typedef struct { double hi, lo; } dd;

static inline dd two_sum(double a, double b) {
    double s = a + b, bb = s - a;
    dd r = {s, (a - (s - bb)) + (b - bb)};
    return r;
}

static inline dd dd_add_prod(dd acc, double x, double y) {
    double p = x * y, pe = fma(x, y, -p);   /* x*y == p + pe exactly */
    dd s = two_sum(acc.hi, p);
    double lo = s.lo + acc.lo + pe;
    dd r = two_sum(s.hi, lo);
    return r;
}

static inline dd dd_sub_prod(dd acc, double x, double y) { return dd_add_prod(acc, -x, y); }

static int dd_threads(void) {
    int n = omp_get_num_procs();
    return n > 0 ? n : 1;
}

/* Real: C[r, c] for r in rows[], c in cols[] -> out[ri * ncols + ci]. */
#define DEFINE_DD_REAL(SUF, T)                                                      \
void dd_gemm_##SUF##_sampled(size_t m, size_t n, size_t k, const T *a,             \
                             const T *b, const int64_t *rows, size_t nrows,         \
                             const int64_t *cols, size_t ncols, double *out_hi,     \
                             double *out_lo) {                                      \
    (void)m;                                                                        \
    _Pragma("omp parallel for schedule(dynamic, 1) num_threads(dd_threads())")      \
    for (size_t ri = 0; ri < nrows; ri++) {                                         \
        const T *ar = a + (size_t)rows[ri] * k;                                     \
        for (size_t ci = 0; ci < ncols; ci++) {                                     \
            dd acc = {0.0, 0.0};                                                    \
            size_t cc = (size_t)cols[ci];                                           \
            for (size_t p = 0; p < k; p++)                                          \
                acc = dd_add_prod(acc, (double)ar[p], (double)b[p * n + cc]);       \
            out_hi[ri * ncols + ci] = acc.hi;                                       \
            if (out_lo) out_lo[ri * ncols + ci] = acc.lo;                           \
        }                                                                           \
    }                                                                               \
}

DEFINE_DD_REAL(f64, double)
DEFINE_DD_REAL(f32, float)

/* Complex interleaved: out has 2 doubles (re, im) per sampled element. */
#define DEFINE_DD_COMPLEX(SUF, T)                                                   \
void dd_gemm_##SUF##_sampled(size_t m, size_t n, size_t k, const T *a,             \
                             const T *b, const int64_t *rows, size_t nrows,         \
                             const int64_t *cols, size_t ncols, double *out) {      \
    (void)m;                                                                        \
    _Pragma("omp parallel for schedule(dynamic, 1) num_threads(dd_threads())")      \
    for (size_t ri = 0; ri < nrows; ri++) {                                         \
        const T *ar = a + 2 * (size_t)rows[ri] * k;                                 \
        for (size_t ci = 0; ci < ncols; ci++) {                                     \
            dd re = {0.0, 0.0}, im = {0.0, 0.0};                                    \
            size_t cc = (size_t)cols[ci];                                           \
            for (size_t p = 0; p < k; p++) {                                        \
                double xr = ar[2 * p], xi = ar[2 * p + 1];                          \
                double yr = b[2 * (p * n + cc)], yi = b[2 * (p * n + cc) + 1];      \
                re = dd_add_prod(re, xr, yr);                                       \
                re = dd_sub_prod(re, xi, yi);                                       \
                im = dd_add_prod(im, xr, yi);                                       \
                im = dd_add_prod(im, xi, yr);                                       \
            }                                                                       \
            out[2 * (ri * ncols + ci)] = re.hi;                                     \
            out[2 * (ri * ncols + ci) + 1] = im.hi;                                 \
        }                                                                           \
    }                                                                               \
}

DEFINE_DD_COMPLEX(c128, double)
DEFINE_DD_COMPLEX(c64, float)

/* Frobenius norm of a (real or complex: pass the interleaved length). */
#define DEFINE_FRO(SUF, T)                                                          \
double dd_fro_##SUF(const T *x, size_t len) {                                      \
    double s = 0.0, scale = 0.0;                                                    \
    /* two-pass with scaling to stay clear of overflow for spread operands */     \
    for (size_t i = 0; i < len; i++) {                                              \
        double v = fabs((double)x[i]);                                              \
        if (v > scale) scale = v;                                                   \
    }                                                                               \
    if (scale == 0.0) return 0.0;                                                   \
    _Pragma("omp parallel for reduction(+ : s) num_threads(dd_threads())")          \
    for (size_t i = 0; i < len; i++) {                                              \
        double v = (double)x[i] / scale;                                            \
        s += v * v;                                                                 \
    }                                                                               \
    return scale * sqrt(s);                                                         \
}

DEFINE_FRO(f64, double)
DEFINE_FRO(f32, float)

/* Sampled normwise error.  `got` holds the candidate's values at the
 * sampled elements (same layout as the dd output, `vals_per_elem` = 1 for
 * real, 2 for complex), `ref` the dd values.  Returns
 * sqrt(sum |got-ref|^2 * (m*n)/(nsamples)) / (||A||_F ||B||_F). */
double dd_normwise(const double *got, const double *ref, size_t nsamp_vals,
                   size_t vals_per_elem, size_t m, size_t n, double norm_a,
                   double norm_b) {
    double s = 0.0, scale = 0.0;
    for (size_t i = 0; i < nsamp_vals; i++) {
        double d = fabs(got[i] - ref[i]);
        if (d > scale) scale = d;
    }
    if (scale == 0.0) return 0.0;
    for (size_t i = 0; i < nsamp_vals; i++) {
        double d = (got[i] - ref[i]) / scale;
        s += d * d;
    }
    double nelem = (double)nsamp_vals / (double)vals_per_elem;
    double fro = scale * sqrt(s * ((double)m * (double)n / nelem));
    return fro / (norm_a * norm_b);
}
