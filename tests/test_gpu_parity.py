"""GPU parity: every GEMM entry point of the C ABI against the oracle.

Integer paths must be bit-exact against the restatement of ferray's CPU GEMM
(oracle/ferray_cpu.c).  Floating-point paths are judged by the normwise error
||C - C_ref||_F / (||A||_F ||B||_F) against the double-double oracle
(oracle/dd_oracle.c) with these tolerances:

* plain f64 / c64:  K * 2^-53 (2K * 2^-53 complex) -- the deterministic
  gamma_K bound of any recursive or blocked dot product;
* plain f32 / c32:  K * 2^-24 (2K * 2^-24 complex);
* split f32 / c32 (3xBF16): 2^-15 + K * 2^-24 -- the dropped lo*lo term and
  the bf16 rounding of lo are each below 2^-16 |a||b| per product;
and, at sizes where it is cheap, the GPU error must not exceed twice the
error of ferray's own CPU result (restated) plus a floor of 2^-50 (f64) /
2^-21 (f32).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

U64, U32 = 2.0 ** -53, 2.0 ** -24

SHAPES = [(1, 1, 1), (17, 13, 9), (64, 64, 64), (128, 256, 128), (300, 257, 129),
          (513, 257, 300), (1024, 1024, 1024)]


def rng(seed=0):
    return np.random.default_rng(seed)


def _err(oracle, a, b, c):
    return oracle.error_vs_dd(a, b, c)


# --------------------------------------------------------------- integers
@pytest.mark.parametrize("m,n,k", SHAPES + [(5, 300, 1000), (129, 65, 4100)])
def test_i8_signed_bit_exact(fg, oracle, m, n, k):
    r = rng(m * 7 + n)
    a = r.integers(-128, 128, (m, k), dtype=np.int8)
    b = r.integers(-128, 128, (k, n), dtype=np.int8)
    c = np.zeros((m, n), np.int32)
    assert fg.gemm_i8_signed(m, n, k, a, b, c)
    np.testing.assert_array_equal(c, oracle.gemm_i8_signed(a, b))


@pytest.mark.parametrize("m,n,k", [(17, 13, 9), (128, 256, 128), (300, 257, 129)])
def test_i8_signed_accumulate(fg, oracle, m, n, k):
    r = rng(3)
    a = r.integers(-128, 128, (m, k), dtype=np.int8)
    b = r.integers(-128, 128, (k, n), dtype=np.int8)
    c0 = r.integers(-2 ** 31, 2 ** 31, (m, n), dtype=np.int64).astype(np.int32)
    c = c0.copy()
    assert fg.gemm_i8_signed(m, n, k, a, b, c, accumulate=True)
    np.testing.assert_array_equal(c, oracle.gemm_i8_signed(a, b, c=c0, accumulate=True))


@pytest.mark.parametrize("m,n,k", SHAPES)
def test_u8i8_bit_exact_vnni(fg, oracle, m, n, k):
    r = rng(m + 11 * n)
    a = r.integers(0, 256, (m, k), dtype=np.uint8)
    b = r.integers(-128, 128, (k, n), dtype=np.int8)
    c = np.zeros((m, n), np.int32)
    assert fg.gemm_i8(m, n, k, a, b, c)
    np.testing.assert_array_equal(c, oracle.gemm_i8(a, b, variant="vnni"))


def test_u8i8_matches_default_avx2_build_without_saturation(fg, oracle):
    # With a < 128 no (k, k+1) pair sum leaves int16, so the default AVX2
    # build's vpmaddubsw saturation never triggers and both builds agree.
    r = rng(5)
    m, n, k = 96, 80, 200
    a = r.integers(0, 128, (m, k), dtype=np.uint8)
    b = r.integers(-128, 128, (k, n), dtype=np.int8)
    c = np.zeros((m, n), np.int32)
    assert fg.gemm_i8(m, n, k, a, b, c)
    np.testing.assert_array_equal(c, oracle.gemm_i8(a, b, variant="avx2"))


@pytest.mark.parametrize("m,n,k", SHAPES + [(33, 70, 3000)])
def test_i16_bit_exact(fg, oracle, m, n, k):
    r = rng(m * 3 + k)
    a = r.integers(-32768, 32768, (m, k), dtype=np.int16)
    b = r.integers(-32768, 32768, (k, n), dtype=np.int16)
    c = np.zeros((m, n), np.int32)
    assert fg.gemm_i16(m, n, k, a, b, c)
    np.testing.assert_array_equal(c, oracle.gemm_i16(a, b))


def test_i16_extremes_wrap(fg, oracle):
    m, n, k = 40, 48, 64
    a = np.full((m, k), -32768, np.int16)
    b = np.full((k, n), -32768, np.int16)
    c = np.zeros((m, n), np.int32)
    assert fg.gemm_i16(m, n, k, a, b, c)
    np.testing.assert_array_equal(c, oracle.gemm_i16(a, b))


def test_integer_golden_cases(fg, oracle):
    import json, os
    cases = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "integer_cases.json")))
    for cs in cases:
        m, n, k = cs["m"], cs["n"], cs["k"]
        if cs["kind"] in ("i16", "i8s"):
            dt = np.int16 if cs["kind"] == "i16" else np.int8
            a = np.array(cs["a"], dt).reshape(m, k)
            b = np.array(cs["b"], dt).reshape(k, n)
            c = np.zeros((m, n), np.int32) if cs["c0"] is None else np.array(cs["c0"], np.int32).reshape(m, n)
            fn = fg.gemm_i16 if cs["kind"] == "i16" else fg.gemm_i8_signed
            assert fn(m, n, k, a, b, c, accumulate=cs["c0"] is not None)
            np.testing.assert_array_equal(c.reshape(-1), np.array(cs["expected"], np.int32), cs["name"])
        else:
            a = np.array(cs["a"], np.uint8).reshape(m, k)
            b = np.array(cs["b"], np.int8).reshape(k, n)
            c0 = cs.get("c0_f32")
            c = np.zeros((m, n), np.float32) if c0 is None else np.array(c0, np.float32).reshape(m, n)
            want = oracle.quantized_matmul(a, cs["a_zp"], cs["scale_a"], b, cs["b_zp"], cs["scale_b"],
                                           c=None if c0 is None else c.copy(), accumulate=c0 is not None)
            assert fg.quantized_matmul(m, n, k, a, cs["a_zp"], np.float32(cs["scale_a"]), b, cs["b_zp"],
                                       np.float32(cs["scale_b"]), c, accumulate=c0 is not None)
            np.testing.assert_array_equal(c, want, cs["name"])


# (40000, 48, 40): more rows than one capped launch of the row-sum kernel has
# warps, so rows past 32768 must still get their own sums.
@pytest.mark.parametrize("m,n,k", [(17, 13, 9), (256, 512, 384), (300, 257, 129), (40000, 48, 40)])
def test_quantized_matmul_bit_exact(fg, oracle, m, n, k):
    r = rng(9)
    a = r.integers(0, 256, (m, k), dtype=np.uint8)
    b = r.integers(-128, 128, (k, n), dtype=np.int8)
    c = np.zeros((m, n), np.float32)
    assert fg.quantized_matmul(m, n, k, a, 7, np.float32(0.01), b, -3, np.float32(0.02), c)
    want = oracle.quantized_matmul(a, 7, 0.01, b, -3, 0.02)
    np.testing.assert_array_equal(c, want)


# --------------------------------------------------------------- floats
@pytest.mark.parametrize("m,n,k", SHAPES)
def test_f64_plain(fg, oracle, m, n, k):
    r = rng(m + n + k)
    a = r.uniform(-1, 1, (m, k))
    b = r.uniform(-1, 1, (k, n))
    c = np.zeros((m, n))
    assert fg.gemm_f64(m, n, k, 1.0, a, b, 0.0, c)
    err = _err(oracle, a, b, c)
    assert err <= k * U64, err
    if m * n * k <= 2 ** 27:
        ref_err = _err(oracle, a, b, oracle.gemm_f64(a, b))
        assert err <= 2 * ref_err + 2.0 ** -50, (err, ref_err)


def test_f64_alpha_beta(fg, oracle):
    r = rng(1)
    m, n, k = 200, 150, 300
    a, b = r.uniform(-1, 1, (m, k)), r.uniform(-1, 1, (k, n))
    c0 = r.uniform(-1, 1, (m, n))
    c = c0.copy()
    assert fg.gemm_f64(m, n, k, 0.5, a, b, -2.0, c)
    want = 0.5 * (a @ b) - 2.0 * c0
    assert np.max(np.abs(c - want)) < 1e-12


@pytest.mark.parametrize("m,n,k", SHAPES)
def test_f32_plain(fg, oracle, m, n, k):
    r = rng(m * n + k)
    a = r.standard_normal((m, k)).astype(np.float32)
    b = r.standard_normal((k, n)).astype(np.float32)
    c = np.zeros((m, n), np.float32)
    assert fg.gemm_f32(m, n, k, 1.0, a, b, 0.0, c)
    err = _err(oracle, a, b, c)
    assert err <= k * U32, err
    if m * n * k <= 2 ** 27:
        ref_err = _err(oracle, a, b, oracle.gemm_f32(a, b))
        assert err <= 2 * ref_err + 2.0 ** -21, (err, ref_err)


@pytest.mark.parametrize("m,n,k", SHAPES + [(2048, 2048, 2048)])
def test_f32_split_3xbf16(fg, oracle, m, n, k):
    r = rng(m + 5 * k)
    a = r.standard_normal((m, k)).astype(np.float32)
    b = r.standard_normal((k, n)).astype(np.float32)
    c = np.zeros((m, n), np.float32)
    assert fg.gemm_f32(m, n, k, 1.0, a, b, 0.0, c, mode="split")
    err = _err(oracle, a, b, c)
    assert err <= 2.0 ** -15 + k * U32, err


@pytest.mark.parametrize("m,n,k", [(17, 13, 9), (300, 257, 129), (1024, 1024, 1024),
                                   (2048, 2048, 2048)])
def test_f32_split6_accuracy(fg, oracle, m, n, k):
    # three BF16 slices represent every f32 exactly; six products leave only
    # terms below 2^-26 |a||b| out, so the error is FP32-accumulation level:
    # no worse than twice the plain FFMA kernel's.
    r = rng(m + 7 * k)
    a = r.standard_normal((m, k)).astype(np.float32)
    b = r.standard_normal((k, n)).astype(np.float32)
    c6, cp = np.zeros((m, n), np.float32), np.zeros((m, n), np.float32)
    assert fg.gemm_f32(m, n, k, 1.0, a, b, 0.0, c6, mode="split", bf16_slices=3)
    assert fg.gemm_f32(m, n, k, 1.0, a, b, 0.0, cp)
    e6, ep = _err(oracle, a, b, c6), _err(oracle, a, b, cp)
    assert e6 <= k * U32, e6
    assert e6 <= 2 * ep + 2.0 ** -30, (e6, ep)


def test_f32_split_alpha_beta(fg):
    r = rng(2)
    m, n, k = 130, 300, 77
    a = r.standard_normal((m, k)).astype(np.float32)
    b = r.standard_normal((k, n)).astype(np.float32)
    c0 = r.standard_normal((m, n)).astype(np.float32)
    c = c0.copy()
    assert fg.gemm_f32(m, n, k, 2.0, a, b, 0.5, c, mode="split")
    want = 2.0 * (a.astype(np.float64) @ b) + 0.5 * c0
    assert np.max(np.abs(c - want)) < 1e-3


def _cplx(r, shape, dt):
    return (r.standard_normal(shape) + 1j * r.standard_normal(shape)).astype(dt)


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (17, 13, 9), (128, 96, 200), (257, 129, 300)])
def test_c64_plain(fg, oracle, m, n, k):
    r = rng(k)
    a, b = _cplx(r, (m, k), np.complex128), _cplx(r, (k, n), np.complex128)
    c = np.zeros((m, n), np.complex128)
    assert fg.gemm_c64(m, n, k, 1.0, 0.0, a, b, 0.0, 0.0, c)
    err = _err(oracle, a, b, c)
    assert err <= 2 * k * U64, err
    ref_err = _err(oracle, a, b, oracle.gemm_complex(a, b))
    assert err <= 2 * ref_err + 2.0 ** -50, (err, ref_err)


@pytest.mark.parametrize("m,n,k", [(33, 47, 59), (300, 260, 700)])
def test_c64_real_scalars_dmma_path(fg, m, n, k):
    # real alpha / beta: the real-embedded DMMA path (beta reads C)
    r = rng(m)
    a, b = _cplx(r, (m, k), np.complex128), _cplx(r, (k, n), np.complex128)
    c0 = _cplx(r, (m, n), np.complex128)
    c = c0.copy()
    assert fg.gemm_c64(m, n, k, -0.75, 0.0, a, b, 1.5, 0.0, c)
    want = -0.75 * (a @ b) + 1.5 * c0
    assert np.max(np.abs(c - want)) < 4 * k * U64 * 10


def test_c64_alpha_beta(fg):
    r = rng(4)
    m, n, k = 33, 47, 59
    a, b = _cplx(r, (m, k), np.complex128), _cplx(r, (k, n), np.complex128)
    c0 = _cplx(r, (m, n), np.complex128)
    c = c0.copy()
    assert fg.gemm_c64(m, n, k, 0.5, -1.5, a, b, 2.0, 0.25, c)
    want = (0.5 - 1.5j) * (a @ b) + (2.0 + 0.25j) * c0
    assert np.max(np.abs(c - want)) < 1e-12


@pytest.mark.parametrize("m,n,k", [(17, 13, 9), (128, 96, 200), (257, 129, 300)])
@pytest.mark.parametrize("mode,slices", [("plain", 0), ("split", 2), ("split", 3)])
def test_c32(fg, oracle, m, n, k, mode, slices):
    r = rng(k + 1)
    a, b = _cplx(r, (m, k), np.complex64), _cplx(r, (k, n), np.complex64)
    c = np.zeros((m, n), np.complex64)
    assert fg.gemm_c32(m, n, k, 1.0, 0.0, a, b, 0.0, 0.0, c, mode=mode, bf16_slices=slices)
    err = _err(oracle, a, b, c)
    tol = 2 * k * U32 if (mode == "plain" or slices == 3) else 2.0 ** -15 + 2 * k * U32
    assert err <= tol, err


# --------------------------------------------------------------- matmul
@pytest.mark.parametrize("dt", [np.float64, np.float32, np.complex128, np.int8, np.int16])
@pytest.mark.parametrize("sa,sb", [((5, 7), (7, 3)), ((7,), (7, 4)), ((6, 7), (7,)),
                                   ((2, 1, 5, 7), (3, 7, 4)), ((4, 5, 7), (7, 6)),
                                   ((2, 3, 40, 70), (1, 3, 70, 30)), ((7,), (2, 7, 3))])
def test_matmul_numpy_semantics(fg, dt, sa, sb):
    r = rng(len(sa) * 10 + len(sb))
    if np.issubdtype(dt, np.integer):
        lo, hi = (-128, 128) if dt == np.int8 else (-300, 300)
        a = r.integers(lo, hi, sa).astype(dt)
        b = r.integers(lo, hi, sb).astype(dt)
        want = np.matmul(a.astype(np.int64), b.astype(np.int64)).astype(np.int32)
    elif np.issubdtype(dt, np.complexfloating):
        a, b = _cplx(r, sa, dt), _cplx(r, sb, dt)
        want = np.matmul(a, b)
    else:
        a = r.standard_normal(sa).astype(dt)
        b = r.standard_normal(sb).astype(dt)
        want = np.matmul(a.astype(np.float64), b.astype(np.float64))
    got = fg.matmul(a, b)
    assert got.shape == want.shape
    if np.issubdtype(dt, np.integer):
        np.testing.assert_array_equal(got, want)
    else:
        tol = 1e-4 if dt == np.float32 else 1e-12
        assert np.max(np.abs(got - want)) <= tol * max(1.0, np.max(np.abs(want)))


def test_matmul_errors(fg):
    with pytest.raises(fg.ShapeMismatch):
        fg.matmul(np.ones((3, 4)), np.ones((5, 2)))
    with pytest.raises(fg.ShapeMismatch):
        fg.matmul(np.ones(3), np.ones(3))
    with pytest.raises(fg.BroadcastFailure):
        fg.matmul(np.ones((2, 3, 4)), np.ones((3, 4, 5)))


def test_matmul_golden_numpy_fixture(fg):
    import json, os
    d = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "matmul_numpy.json")))
    for cs in d["cases"]:
        a = np.array(cs["a"], np.float64).reshape(cs["a_shape"])
        b = np.array(cs["b"], np.float64).reshape(cs["b_shape"])
        got = fg.matmul(a, b)
        np.testing.assert_array_equal(got.reshape(-1), np.array(cs["expected"]), cs["name"])


def test_device_resident_matmul(fg):
    r = rng(8)
    a = r.standard_normal((64, 48))
    b = r.standard_normal((48, 80))
    da, db = fg.DeviceArray.from_numpy(a), fg.DeviceArray.from_numpy(b)
    dc = fg.matmul(da, db)
    assert isinstance(dc, fg.DeviceArray)
    assert np.max(np.abs(dc.to_numpy() - a @ b)) < 1e-12


def test_batched_strided_broadcast(fg):
    r = rng(12)
    bsz, m, n, k = 5, 70, 90, 130
    a = r.integers(-128, 128, (bsz, m, k), dtype=np.int8)
    b = r.integers(-128, 128, (k, n), dtype=np.int8)
    da, db = fg.DeviceArray.from_numpy(a), fg.DeviceArray.from_numpy(b)
    dc = fg.DeviceArray((bsz, m, n), np.int32)
    fg.gemm_batched_strided(np.int8, bsz, m, n, k, da, m * k, db, 0, dc, m * n)
    want = np.matmul(a.astype(np.int64), b.astype(np.int64)).astype(np.int32)
    np.testing.assert_array_equal(dc.to_numpy(), want)


# --------------------------------------------------- pipelined host path
def test_host_path_row_panels_i8_exact(fg):
    # 90 MB of operands + result: the host-pointer call streams 2 row panels
    m, n, k = 6000, 3000, 2000
    r = rng(21)
    a = r.integers(-128, 128, (m, k), dtype=np.int8)
    b = r.integers(-128, 128, (k, n), dtype=np.int8)
    c = np.zeros((m, n), np.int32)
    assert fg.gemm_i8_signed(m, n, k, a, b, c)
    want = (a.astype(np.float64) @ b.astype(np.float64)).astype(np.int32)  # exact: |C| < 2^53
    np.testing.assert_array_equal(c, want)
    # accumulate reads C through the panels too
    c0 = r.integers(-2 ** 20, 2 ** 20, (m, n), dtype=np.int32)
    c = c0.copy()
    assert fg.gemm_i8_signed(m, n, k, a, b, c, accumulate=True)
    np.testing.assert_array_equal(c, want + c0)


@pytest.mark.parametrize("mode", ["plain", "split"])
def test_host_path_row_panels_f32_beta(fg, oracle, mode):
    m, n, k = 5000, 3000, 1500
    r = rng(22)
    a = r.standard_normal((m, k), dtype=np.float32)
    b = r.standard_normal((k, n), dtype=np.float32)
    c0 = r.standard_normal((m, n), dtype=np.float32)
    c = c0.copy()
    assert fg.gemm_f32(m, n, k, 1.5, a, b, -0.5, c, mode=mode)
    rows, cols = oracle.sample_indices(m, n, 64, 64, seed=3)
    ref = 1.5 * oracle.dd_sampled(a, b, rows, cols) - 0.5 * c0[np.ix_(rows, cols)].astype(np.float64)
    got = c[np.ix_(rows, cols)]
    scale = np.linalg.norm(a.astype(np.float64)) * np.linalg.norm(b.astype(np.float64))
    blow = np.sqrt(m * n / got.size)  # sampled block -> whole-matrix Frobenius norms
    err = np.linalg.norm(got - ref) * blow / scale
    # GEMM bound plus the rounding of the f32 output (|C| ~ |beta C0| here)
    tol = (2.0 ** -15 if mode == "split" else 0.0) + (k + 4) * U32
    assert err <= tol + 2 * U32 * np.linalg.norm(ref) * blow / scale


def test_host_path_many_panels_i8_exact(fg):
    # 230 MB of operands and result: 4 row panels, the last cut to 256 rows
    m, n, k = 12000, 4096, 2048
    r = rng(23)
    a = r.integers(-128, 128, (m, k), dtype=np.int8)
    b = r.integers(-128, 128, (k, n), dtype=np.int8)
    c0 = r.integers(-2 ** 20, 2 ** 20, (m, n), dtype=np.int32)
    want = (a.astype(np.float64) @ b.astype(np.float64)).astype(np.int64)
    c = c0.copy()
    assert fg.gemm_i8_signed(m, n, k, a, b, c, accumulate=True)
    np.testing.assert_array_equal(c, (want + c0).astype(np.int32))


def test_host_path_many_panels_f32_beta(fg, oracle):
    # 262 MB, beta != 0 (C is read through the panels); n not a power of two
    m, n, k = 12000, 4000, 1024
    r = rng(24)
    a = r.standard_normal((m, k), dtype=np.float32)
    b = r.standard_normal((k, n), dtype=np.float32)
    c0 = r.standard_normal((m, n), dtype=np.float32)
    c = c0.copy()
    assert fg.gemm_f32(m, n, k, 1.5, a, b, -0.5, c)
    rows, cols = oracle.sample_indices(m, n, 64, 64, seed=4)
    cols = np.unique(np.concatenate([cols, [0, 1023, 1024, 3071, 3072, 3999]]))
    ref = 1.5 * oracle.dd_sampled(a, b, rows, cols) - 0.5 * c0[np.ix_(rows, cols)].astype(np.float64)
    got = c[np.ix_(rows, cols)]
    scale = np.linalg.norm(a.astype(np.float64)) * np.linalg.norm(b.astype(np.float64))
    blow = np.sqrt(m * n / got.size)
    err = np.linalg.norm(got - ref) * blow / scale
    assert err <= (k + 4) * U32 + 2 * U32 * np.linalg.norm(ref) * blow / scale


# ------------------------------------------------------------------ GEMV
@pytest.mark.parametrize("dt,u", [(np.float64, U64), (np.float32, U32)])
@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (300, 1, 1001), (8192, 1, 4096), (1, 300, 1001),
                                   (1, 4097, 3000), (1, 200, 100000), (5, 1, 77)])
def test_gemv_shapes(fg, oracle, dt, u, m, n, k):
    r = rng(m + 3 * n + k)
    a = r.uniform(-1, 1, (m, k)).astype(dt)
    b = r.uniform(-1, 1, (k, n)).astype(dt)
    c0 = r.uniform(-1, 1, (m, n)).astype(dt)
    gemm = fg.gemm_f64 if dt == np.float64 else fg.gemm_f32
    c = np.zeros((m, n), dt)
    assert gemm(m, n, k, 1.0, a, b, 0.0, c)
    exact = oracle.dd_full(a, b)
    scale = np.linalg.norm(a.astype(np.float64)) * np.linalg.norm(b.astype(np.float64))
    assert np.linalg.norm(c - exact) / scale <= k * u
    c = c0.copy()
    assert gemm(m, n, k, -0.5, a, b, 1.5, c)
    ref = -0.5 * exact + 1.5 * c0.astype(np.float64)
    assert np.linalg.norm(c - ref) <= (k + 4) * u * scale + 2 * u * np.linalg.norm(ref)


def test_matmul_vector_operands_use_gemv(fg):
    r = rng(8)
    a = r.standard_normal((513, 700))
    v = r.standard_normal(700)
    w = r.standard_normal(513)
    da, dv, dw = (fg.DeviceArray.from_numpy(x) for x in (a, v, w))
    got = fg.matmul(da, dv).to_numpy()
    np.testing.assert_allclose(got, a @ v, rtol=0, atol=700 * U64 * 30)
    got = fg.matmul(dw, da).to_numpy()
    np.testing.assert_allclose(got, w @ a, rtol=0, atol=513 * U64 * 30)


# ------------------------------------------------------- bf16 / f16 -> f32
def _bf16_bits(x):
    """round-to-nearest-even f32 -> bf16 bit patterns"""
    u = x.astype(np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return u.astype(np.uint16)


@pytest.mark.parametrize("kind", ["bf16", "f16"])
@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (17, 13, 9), (128, 256, 128), (300, 257, 1000),
                                   (513, 300, 2048), (1024, 1024, 1024)])
def test_half_gemm_f32(fg, oracle, kind, m, n, k):
    r = rng(m + n + k)
    af, bf = r.standard_normal((m, k)), r.standard_normal((k, n))
    if kind == "bf16":
        a, b = _bf16_bits(af), _bf16_bits(bf)
        aw, bw = oracle.bf16_to_f32(a), oracle.bf16_to_f32(b)
        gemm, ref = fg.gemm_bf16_f32, oracle.gemm_bf16_f32
    else:
        a, b = af.astype(np.float16), bf.astype(np.float16)
        aw, bw = a.astype(np.float32), b.astype(np.float32)
        gemm, ref = fg.gemm_f16_f32, oracle.gemm_f16_f32
    c = np.zeros((m, n), np.float32)
    assert gemm(m, n, k, a, b, c)
    err = _err(oracle, aw, bw, c)
    assert err <= k * U32, err
    ref_err = _err(oracle, aw, bw, ref(a, b))
    assert err <= 2 * ref_err + 2.0 ** -21, (err, ref_err)
    # accumulate: C += A @ B
    c0 = r.standard_normal((m, n)).astype(np.float32)
    c = c0.copy()
    assert gemm(m, n, k, a, b, c, accumulate=True)
    want = oracle.dd_full(aw, bw) + c0.astype(np.float64)
    scale = np.linalg.norm(aw.astype(np.float64)) * np.linalg.norm(bw.astype(np.float64))
    assert np.linalg.norm(c - want) <= (k + 4) * U32 * scale + 2 * U32 * np.linalg.norm(want)


@pytest.mark.parametrize("variant,splits", [(0, 1), (2, 1), (0, 4), (2, 3)])
def test_half_gemm_tile_variants(fg, oracle, variant, splits):
    r = rng(5)
    m, n, k = 300, 260, 3000
    a, b = _bf16_bits(r.standard_normal((m, k))), _bf16_bits(r.standard_normal((k, n)))
    c = np.zeros((m, n), np.float32)
    with fg.tune_forced("split_f32", variant, splits):
        assert fg.gemm_bf16_f32(m, n, k, a, b, c)
    assert _err(oracle, oracle.bf16_to_f32(a), oracle.bf16_to_f32(b), c) <= k * U32
