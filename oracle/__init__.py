"""The oracle: test infrastructure only.

Two C libraries behind ctypes, used by tests/, by __graft_entry__.smoke() and
by bench.py's CPU-baseline leg -- as the checker, never as the product path:

* ``ferray_cpu.c`` restates ferray-linalg's CPU GEMM (every dtype on the
  matmul path, with its summation order and integer saturation rules);
* ``dd_oracle.c`` computes double-double reference results and normwise
  errors ||C - C_ref||_F / (||A||_F ||B||_F).

Parity of the restatement is pinned against the reference's own golden
vectors (tests/golden/, extracted by tests/golden/make_golden.py).
"""
import ctypes as C
import os

import numpy as np

from . import build as _build

_lib = None


def lib():
    global _lib
    if _lib is None:
        path = _build.LIB
        if not os.path.exists(path):
            _build.build()
        _lib = C.CDLL(path)
        _declare(_lib)
    return _lib


_sz = C.c_size_t
_p = C.c_void_p


def _declare(L):
    L.fr_set_threads.argtypes = [C.c_int]
    L.fr_gemm_f64.argtypes = [_sz, _sz, _sz, C.c_double, _p, _p, C.c_double, _p]
    L.fr_gemm_f32.argtypes = [_sz, _sz, _sz, C.c_float, _p, _p, C.c_float, _p]
    L.fr_gemm_c64.argtypes = [_sz, _sz, _sz, C.c_double, C.c_double, _p, _p,
                              C.c_double, C.c_double, _p]
    L.fr_gemm_c32.argtypes = [_sz, _sz, _sz, C.c_float, C.c_float, _p, _p,
                              C.c_float, C.c_float, _p]
    for name in ("fr_gemm_i8_signed", "fr_gemm_i8_signed_rows", "fr_gemm_i16", "fr_gemm_i8_vnni",
                 "fr_gemm_i8_avx2"):
        getattr(L, name).argtypes = [_sz, _sz, _sz, _p, _p, _p, C.c_int]
    L.fr_quantized_matmul.argtypes = [_sz, _sz, _sz, _p, C.c_uint8, C.c_float, _p,
                                      C.c_int8, C.c_float, _p, C.c_int, C.c_int]
    L.fr_pick_grid.argtypes = [_sz, _sz, _sz, _sz, C.c_int, _p, _p]
    L.fr_matmul_raw_f64.argtypes = [_p, _p, _sz, _sz, _sz, _p]
    L.fr_matmul_raw_f32.argtypes = [_p, _p, _sz, _sz, _sz, _p]
    for name in ("dd_gemm_f64_sampled", "dd_gemm_f32_sampled"):
        getattr(L, name).argtypes = [_sz, _sz, _sz, _p, _p, _p, _sz, _p, _sz, _p, _p]
    for name in ("dd_gemm_c128_sampled", "dd_gemm_c64_sampled"):
        getattr(L, name).argtypes = [_sz, _sz, _sz, _p, _p, _p, _sz, _p, _sz, _p]
    L.dd_fro_f64.argtypes = [_p, _sz]
    L.dd_fro_f64.restype = C.c_double
    L.dd_fro_f32.argtypes = [_p, _sz]
    L.dd_fro_f32.restype = C.c_double
    L.dd_normwise.argtypes = [_p, _p, _sz, _sz, _sz, _sz, C.c_double, C.c_double]
    L.dd_normwise.restype = C.c_double


def _ptr(x):
    return x.ctypes.data_as(C.c_void_p)


def set_threads(n):
    lib().fr_set_threads(int(n))


# --------------------------------------------------------------------------
# ferray CPU GEMM restatement (numpy in, numpy out)
# --------------------------------------------------------------------------

def gemm_f64(a, b, alpha=1.0, beta=0.0, c=None):
    m, k = a.shape
    n = b.shape[1]
    a = np.ascontiguousarray(a, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    c = np.zeros((m, n), np.float64) if c is None else np.array(c, np.float64, order="C")
    lib().fr_gemm_f64(m, n, k, alpha, _ptr(a), _ptr(b), beta, _ptr(c))
    return c


def gemm_f32(a, b, alpha=1.0, beta=0.0, c=None):
    m, k = a.shape
    n = b.shape[1]
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    c = np.zeros((m, n), np.float32) if c is None else np.array(c, np.float32, order="C")
    lib().fr_gemm_f32(m, n, k, alpha, _ptr(a), _ptr(b), beta, _ptr(c))
    return c


def chain_order(dims):
    """products/mod.rs:839-855: optimal chain parenthesisation, u64 costs,
    the first k reaching the minimum wins; split[i][j] = k."""
    n = len(dims) - 1
    cost = [[0] * n for _ in range(n)]
    split = [[0] * n for _ in range(n)]
    for length in range(2, n + 1):
        for i in range(0, n - length + 1):
            j = i + length - 1
            cost[i][j] = 2 ** 64 - 1
            for k in range(i, j):
                q = cost[i][k] + cost[k + 1][j] + dims[i] * dims[k + 1] * dims[j + 1]
                if q < cost[i][j]:
                    cost[i][j] = q
                    split[i][j] = k
    return np.array(split, dtype=np.int64)


def multi_dot(arrays):
    """products/mod.rs:858-902: multiply along chain_order with the restated
    GEMM (f64 / f32 by dtype)."""
    dims = [arrays[0].shape[0]] + [x.shape[1] for x in arrays]
    split = chain_order(dims)
    mm = gemm_f64 if arrays[0].dtype == np.float64 else gemm_f32

    def prod(i, j):
        if i == j:
            return arrays[i]
        k = split[i][j]
        return mm(prod(i, k), prod(k + 1, j))
    return prod(0, len(arrays) - 1)


def matrix_power(a, n):
    """solve.rs:478-491 for n > 0: result = I; result @= base on set bits;
    base = base @ base (the restated GEMM)."""
    mm = gemm_f64 if a.dtype == np.float64 else gemm_f32
    result = np.eye(a.shape[0], dtype=a.dtype)
    base = a.copy()
    p = n
    while p > 0:
        if p & 1:
            result = mm(result, base)
        base = mm(base, base)
        p >>= 1
    return result


def tensordot(a, b, axes_a, axes_b):
    """products/tensordot.rs:86-153: permute a (free axes, then contracted)
    and b (contracted, then free), then the naive loop sum += x * y in k
    order (separate multiply and add, the Rust `+=` of a product)."""
    fa = [i for i in range(a.ndim) if i not in axes_a]
    fb = [i for i in range(b.ndim) if i not in axes_b]
    ap = np.transpose(a, fa + list(axes_a)).reshape(int(np.prod([a.shape[i] for i in fa])), -1)
    bp = np.transpose(b, list(axes_b) + fb).reshape(ap.shape[1], -1)
    out = np.zeros((ap.shape[0], bp.shape[1]), a.dtype)
    for k in range(ap.shape[1]):
        out = out + ap[:, k:k + 1] * bp[k:k + 1, :]
    return out.reshape([a.shape[i] for i in fa] + [b.shape[i] for i in fb])


_TRSM_NB = 32  # trsm.rs:33


def trsm_left(a, b, alpha=1.0, upper=False, unit_diag=False):
    """ferray-linalg/src/trsm.rs:46-133 restated: X with op(A) X = alpha B
    (a m x m, b m x n; b is copied, its dtype kept).  The same alpha scale
    (trsm.rs:137-153), block recursion and split rule (trsm.rs:165-200,
    264-300), unblocked substitution (trsm.rs:227-262, 304-332) and scalar
    trailing update (trsm.rs:205-225), vectorised over columns only: every
    element sees the reference's operations in the reference's order (a
    product, then a difference; 1 / a_ii, then a product; no fused
    multiply-add)."""
    t = a.dtype.type
    x = np.array(b, copy=True)
    m, n = x.shape
    if m == 0 or n == 0:
        return x
    if alpha != 1.0:
        x *= t(alpha)

    def unblocked(r0, mm):
        for i in (range(mm - 1, -1, -1) if upper else range(mm)):
            for p in (range(i + 1, mm) if upper else range(i)):
                x[r0 + i] -= a[r0 + i, r0 + p] * x[r0 + p]
            if not unit_diag:
                x[r0 + i] *= t(1) / a[r0 + i, r0 + i]

    def update(d0, rows, s0, blk):  # x[d0:d0+rows] -= blk @ x[s0:...], p ascending
        for p in range(blk.shape[1]):
            x[d0:d0 + rows] -= blk[:, p:p + 1] * x[s0 + p][None, :]

    def rec(r0, mm):
        if mm <= _TRSM_NB:
            unblocked(r0, mm)
            return
        m1 = min(-(-(mm // 2) // _TRSM_NB) * _TRSM_NB, mm - _TRSM_NB)
        m2 = mm - m1
        if not upper:
            rec(r0, m1)
            update(r0 + m1, m2, r0, a[r0 + m1:r0 + mm, r0:r0 + m1])
            rec(r0 + m1, m2)
        else:
            rec(r0 + m1, m2)
            update(r0, m1, r0 + m1, a[r0:r0 + m1, r0 + m1:r0 + mm])
            rec(r0, m1)

    rec(0, m)
    return x


def trsm_test_triangle(m, upper=False):
    """The triangular test matrices of trsm.rs:492-518: diagonal
    2 + 0.5 i, off-diagonal 0.1 (i + j + 1) on the stored triangle."""
    i, j = np.indices((m, m))
    a = np.where(i == j, 2.0 + 0.5 * i, 0.1 * (i + j + 1))
    keep = (j >= i) if upper else (j <= i)
    return np.where(keep, a, 0.0)


def bf16_to_f32(bits):
    """bf16 bit patterns (uint16) -> f32, exact (the `half` crate's widening)."""
    return (np.asarray(bits, np.uint16).astype(np.uint32) << 16).view(np.float32)


def gemm_bf16_f32(a_bits, b_bits, c=None, accumulate=False):
    """gemm/mod.rs:851-882: widen both bf16 operands to f32 (exact), then the
    SGEMM with beta = 1 when accumulating, 0 otherwise."""
    return gemm_f32(bf16_to_f32(a_bits), bf16_to_f32(b_bits), 1.0, 1.0 if accumulate else 0.0, c)


def gemm_f16_f32(a, b, c=None, accumulate=False):
    """gemm/mod.rs:906-933: widen f16 -> f32 (exact), then the SGEMM."""
    a = np.asarray(a, np.float16).astype(np.float32)
    b = np.asarray(b, np.float16).astype(np.float32)
    return gemm_f32(a, b, 1.0, 1.0 if accumulate else 0.0, c)


def gemm_complex(a, b, alpha=1.0 + 0j, beta=0j, c=None):
    """c64 (complex128) or c32 (complex64) according to a.dtype."""
    m, k = a.shape
    n = b.shape[1]
    dt = np.complex128 if a.dtype == np.complex128 else np.complex64
    a = np.ascontiguousarray(a, dt)
    b = np.ascontiguousarray(b, dt)
    c = np.zeros((m, n), dt) if c is None else np.array(c, dt, order="C")
    fn = lib().fr_gemm_c64 if dt == np.complex128 else lib().fr_gemm_c32
    fn(m, n, k, alpha.real, alpha.imag, _ptr(a), _ptr(b), beta.real, beta.imag, _ptr(c))
    return c


def _int_gemm(name, a, b, c, accumulate):
    m, k = a.shape
    n = b.shape[1]
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    c = np.zeros((m, n), np.int32) if c is None else np.array(c, np.int32, order="C")
    getattr(lib(), name)(m, n, k, _ptr(a), _ptr(b), _ptr(c), int(bool(accumulate)))
    return c


def gemm_i8_signed(a, b, c=None, accumulate=False):
    return _int_gemm("fr_gemm_i8_signed", a.astype(np.int8, copy=False),
                     b.astype(np.int8, copy=False), c, accumulate)


def gemm_i8_signed_rows(a, b, c=None, accumulate=False):
    """The same product as gemm_i8_signed by a plain row loop (exact sums,
    no packing): the cross-check for the packed restatement."""
    return _int_gemm("fr_gemm_i8_signed_rows", a.astype(np.int8, copy=False),
                     b.astype(np.int8, copy=False), c, accumulate)


def pick_grid(m, n, k, workers, f32=False):
    """(parallel, mw, nw): the thread grid ferray's GEMM driver picks
    (gemm/outer.rs:343-383, 692-726)."""
    mw, nw = C.c_size_t(), C.c_size_t()
    par = lib().fr_pick_grid(m, n, k, workers, int(bool(f32)), C.byref(mw), C.byref(nw))
    return bool(par), mw.value, nw.value


def gemm_i16(a, b, c=None, accumulate=False):
    return _int_gemm("fr_gemm_i16", a.astype(np.int16, copy=False),
                     b.astype(np.int16, copy=False), c, accumulate)


def gemm_i8(a, b, c=None, accumulate=False, variant="vnni"):
    """u8 x i8.  variant 'vnni' (exact; avxvnni/avx512 builds) or 'avx2'
    (default build: int16 saturation of adjacent K pairs in full tiles)."""
    name = "fr_gemm_i8_vnni" if variant == "vnni" else "fr_gemm_i8_avx2"
    return _int_gemm(name, a.astype(np.uint8, copy=False), b.astype(np.int8, copy=False),
                     c, accumulate)


def quantized_matmul(a, a_zp, scale_a, b, b_zp, scale_b, c=None, accumulate=False,
                     variant="vnni"):
    m, k = a.shape
    n = b.shape[1]
    a = np.ascontiguousarray(a, np.uint8)
    b = np.ascontiguousarray(b, np.int8)
    c = np.zeros((m, n), np.float32) if c is None else np.array(c, np.float32, order="C")
    lib().fr_quantized_matmul(m, n, k, _ptr(a), a_zp, scale_a, _ptr(b), b_zp, scale_b,
                              _ptr(c), int(bool(accumulate)), int(variant == "vnni"))
    return c


def matmul_raw(a, b):
    m, k = a.shape
    n = b.shape[1]
    if a.dtype == np.float64:
        out = np.empty((m, n), np.float64)
        lib().fr_matmul_raw_f64(_ptr(np.ascontiguousarray(a)), _ptr(np.ascontiguousarray(b)),
                                m, k, n, _ptr(out))
    else:
        out = np.empty((m, n), np.float32)
        lib().fr_matmul_raw_f32(_ptr(np.ascontiguousarray(a, np.float32)),
                                _ptr(np.ascontiguousarray(b, np.float32)), m, k, n, _ptr(out))
    return out


# --------------------------------------------------------------------------
# double-double oracle
# --------------------------------------------------------------------------

def dd_sampled(a, b, rows, cols):
    """DD reference of (a @ b)[rows][:, cols] as float64 (complex128 for
    complex operands)."""
    m, k = a.shape
    n = b.shape[1]
    rows = np.ascontiguousarray(rows, np.int64)
    cols = np.ascontiguousarray(cols, np.int64)
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    L = lib()
    if np.iscomplexobj(a):
        out = np.empty((len(rows), len(cols)), np.complex128)
        fn = L.dd_gemm_c128_sampled if a.dtype == np.complex128 else L.dd_gemm_c64_sampled
        fn(m, n, k, _ptr(a), _ptr(b), _ptr(rows), len(rows), _ptr(cols), len(cols), _ptr(out))
        return out
    hi = np.empty((len(rows), len(cols)), np.float64)
    fn = L.dd_gemm_f64_sampled if a.dtype == np.float64 else L.dd_gemm_f32_sampled
    fn(m, n, k, _ptr(a), _ptr(b), _ptr(rows), len(rows), _ptr(cols), len(cols), _ptr(hi), None)
    return hi


def dd_full(a, b):
    return dd_sampled(a, b, np.arange(a.shape[0]), np.arange(b.shape[1]))


def fro(x):
    x = np.ascontiguousarray(x)
    if np.iscomplexobj(x):
        x = x.view(np.float64 if x.dtype == np.complex128 else np.float32)
    if x.dtype == np.float64:
        return lib().dd_fro_f64(_ptr(x), x.size)
    x = np.ascontiguousarray(x, np.float32)
    return lib().dd_fro_f32(_ptr(x), x.size)


def sample_indices(m, n, max_rows=256, max_cols=256, seed=1234):
    """Seeded row/column sample (all of them when small)."""
    rng = np.random.default_rng(seed)
    rows = np.arange(m) if m <= max_rows else np.sort(rng.choice(m, max_rows, replace=False))
    cols = np.arange(n) if n <= max_cols else np.sort(rng.choice(n, max_cols, replace=False))
    return rows, cols


def normwise_error(got_sampled, ref_sampled, m, n, norm_a, norm_b):
    """||C - C_ref||_F / (||A||_F ||B||_F) estimated on the sampled block."""
    g = np.ascontiguousarray(got_sampled)
    r = np.ascontiguousarray(ref_sampled)
    vpe = 1
    if np.iscomplexobj(r) or np.iscomplexobj(g):
        g = np.ascontiguousarray(g, np.complex128).view(np.float64)
        r = np.ascontiguousarray(r, np.complex128).view(np.float64)
        vpe = 2
    else:
        g = np.ascontiguousarray(g, np.float64)
        r = np.ascontiguousarray(r, np.float64)
    return lib().dd_normwise(_ptr(g), _ptr(r), g.size, vpe, m, n, norm_a, norm_b)


def error_vs_dd(a, b, c, rows=None, cols=None):
    """Normwise error of candidate result c against the DD oracle."""
    m, n = c.shape
    if rows is None:
        rows, cols = sample_indices(m, n)
    ref = dd_sampled(a, b, rows, cols)
    got = c[np.ix_(rows, cols)]
    return normwise_error(got, ref, m, n, fro(a), fro(b))
