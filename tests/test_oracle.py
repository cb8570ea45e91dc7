"""CPU tests of the oracle itself, pinned to the reference's golden vectors.

* ferray's restated CPU GEMM reproduces the NumPy 2.4.5 fixture
  (fixtures/linalg/matmul.json, tolerance_ulps per case) and the exact NumPy
  hex-float answers of gemm/mod.rs:1213-1275;
* the integer restatement equals the naive wrapping-i32 loops the reference
  asserts against (gemm/integer_tests.rs), case by case;
* the double-double oracle agrees with exact rational arithmetic on small
  cases and is far more accurate than any FP64 result it judges.
"""
import json
import os
from fractions import Fraction

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def ulps(a, b):
    a = np.asarray(a, np.float64).view(np.int64)
    b = np.asarray(b, np.float64).view(np.int64)
    return np.abs(a - b)


def test_numpy_fixture_matmul(oracle):
    d = json.load(open(os.path.join(GOLD, "matmul_numpy.json")))
    assert d["numpy_version"] == "2.4.5"
    for cs in d["cases"]:
        a = np.array(cs["a"], np.float64).reshape(cs["a_shape"])
        b = np.array(cs["b"], np.float64).reshape(cs["b_shape"])
        exp = np.array(cs["expected"], np.float64)
        got = oracle.matmul_raw(a, b).reshape(-1)
        # ferray-test-oracle floors every ULP tolerance at 10 (lib.rs:59)
        assert np.all(ulps(got, exp) <= max(cs["tolerance_ulps"], 10)), cs["name"]
        dd = oracle.dd_full(a, b).reshape(-1)
        assert np.all(ulps(dd, exp) <= cs["tolerance_ulps"]), cs["name"]


def test_hexfloat_goldens(oracle):
    cases = json.load(open(os.path.join(GOLD, "gemm_hexfloat.json")))
    for cs in cases:
        a = np.array([float.fromhex(x) for x in cs["a"]]).reshape(cs["a_shape"])
        b = np.array([float.fromhex(x) for x in cs["b"]]).reshape(cs["b_shape"])
        exp = np.array([float.fromhex(x) for x in cs["expected"]])
        got = oracle.gemm_f64(a, b).reshape(-1)
        assert np.all(ulps(got, exp) <= cs["max_ulps"]), (cs["name"], got, exp)
        # NumPy's answer itself carries rounding error (up to k*u*|A||B|
        # elementwise), so the correctly rounded DD value may differ from it
        # by more ulps where the sum cancels; bound the difference instead.
        dd = oracle.dd_full(a, b).reshape(-1)
        bound = (np.abs(a) @ np.abs(b)).reshape(-1) * a.shape[1] * 2.0 ** -53
        assert np.all(np.abs(dd - exp) <= bound), cs["name"]


def test_integer_golden_cases(oracle):
    cases = json.load(open(os.path.join(GOLD, "integer_cases.json")))
    seen = set()
    for cs in cases:
        m, n, k = cs["m"], cs["n"], cs["k"]
        seen.add(cs["kind"])
        if cs["kind"] in ("i16", "i8s"):
            dt = np.int16 if cs["kind"] == "i16" else np.int8
            a = np.array(cs["a"], dt).reshape(m, k)
            b = np.array(cs["b"], dt).reshape(k, n)
            c0 = None if cs["c0"] is None else np.array(cs["c0"], np.int32).reshape(m, n)
            fn = oracle.gemm_i16 if cs["kind"] == "i16" else oracle.gemm_i8_signed
            got = fn(a, b, c=c0, accumulate=c0 is not None)
            np.testing.assert_array_equal(got.reshape(-1), np.array(cs["expected"], np.int32),
                                          cs["name"])
        else:
            a = np.array(cs["a"], np.uint8).reshape(m, k)
            b = np.array(cs["b"], np.int8).reshape(k, n)
            c0 = cs.get("c0_f32")
            c0 = None if c0 is None else np.array(c0, np.float32).reshape(m, n)
            # the naive formula of integer_tests.rs:30-63
            acc = ((a.astype(np.int64) - cs["a_zp"]) @ (b.astype(np.int64) - cs["b_zp"]))
            acc = ((acc + 2 ** 31) % 2 ** 32 - 2 ** 31).astype(np.int32)
            want = np.float32(np.float32(cs["scale_a"]) * np.float32(cs["scale_b"])) * acc.astype(np.float32)
            if c0 is not None:
                want = c0 + want
            for variant in ("vnni", "avx2"):
                got = oracle.quantized_matmul(a, cs["a_zp"], cs["scale_a"], b, cs["b_zp"],
                                              cs["scale_b"], c=None if c0 is None else c0.copy(),
                                              accumulate=c0 is not None, variant=variant)
                rel = np.abs(got - want) / np.maximum(np.abs(want), 1.0)
                assert np.all(rel < cs["rel_tol"]), (cs["name"], variant)
    assert seen == {"i16", "i8s", "qmm"}


def test_u8i8_avx2_saturates_only_full_tiles(oracle):
    # a = 255 and b = 127 on a K pair: 2*255*127 = 64770 > 32767 saturates in
    # full 4x8 tiles (kernel_avx2_i8.rs:97-117); the edge tile stays exact.
    m, n, k = 5, 9, 4
    a = np.full((m, k), 255, np.uint8)
    b = np.full((k, n), 127, np.int8)
    exact = oracle.gemm_i8(a, b, variant="vnni")
    sat = oracle.gemm_i8(a, b, variant="avx2")
    assert np.all(exact == 4 * 255 * 127)
    assert np.all(sat[:4, :8] == 2 * 32767)
    assert np.all(sat[4, :] == exact[4, :]) and np.all(sat[:, 8] == exact[:, 8])


def test_dd_exact_small(oracle):
    rng = np.random.default_rng(0)
    a = rng.uniform(-1, 1, (6, 9))
    b = rng.uniform(-1, 1, (9, 5))
    dd = oracle.dd_full(a, b)
    for i in range(6):
        for j in range(5):
            exact = sum(Fraction(a[i, p]) * Fraction(b[p, j]) for p in range(9))
            assert dd[i, j] == float(exact)


def test_dd_complex_and_f32(oracle):
    rng = np.random.default_rng(1)
    a = (rng.standard_normal((7, 11)) + 1j * rng.standard_normal((7, 11)))
    b = (rng.standard_normal((11, 4)) + 1j * rng.standard_normal((11, 4)))
    dd = oracle.dd_full(a, b)
    assert np.max(np.abs(dd - a @ b)) < 1e-13
    af = a.astype(np.complex64)
    bf = b.astype(np.complex64)
    ddf = oracle.dd_full(af, bf)
    want = af.astype(np.complex128) @ bf.astype(np.complex128)
    assert np.max(np.abs(ddf - want)) < 1e-13


@pytest.mark.parametrize("m,n,k", [(17, 13, 9), (8, 6, 300), (129, 65, 513)])
def test_restatement_close_to_dd(oracle, m, n, k):
    rng = np.random.default_rng(m)
    a = rng.uniform(-1, 1, (m, k))
    b = rng.uniform(-1, 1, (k, n))
    c = oracle.gemm_f64(a, b)
    assert oracle.error_vs_dd(a, b, c) <= k * 2.0 ** -53
    af, bf = a.astype(np.float32), b.astype(np.float32)
    assert oracle.error_vs_dd(af, bf, oracle.gemm_f32(af, bf)) <= k * 2.0 ** -24


def test_restatement_panel_summation_order(oracle):
    # K = 300 spans two KC=256 panels: C = chain(0..256) + chain(256..300),
    # each chain a fused-multiply-add recurrence from zero (outer.rs:415-421).
    rng = np.random.default_rng(7)
    m, n, k = 8, 16, 300
    a = rng.uniform(-1, 1, (m, k))
    b = rng.uniform(-1, 1, (k, n))
    got = oracle.gemm_f64(a, b)
    import ctypes
    libm = ctypes.CDLL("libm.so.6")
    libm.fma.restype = ctypes.c_double
    libm.fma.argtypes = [ctypes.c_double] * 3
    for i in (0, 5):
        for j in (0, 11):
            p1 = 0.0
            for p in range(256):
                p1 = libm.fma(a[i, p], b[p, j], p1)
            p2 = 0.0
            for p in range(256, 300):
                p2 = libm.fma(a[i, p], b[p, j], p2)
            assert got[i, j] == p1 + p2


def test_alpha_beta_rules(oracle):
    rng = np.random.default_rng(3)
    m, n, k = 9, 17, 20
    a, b = rng.uniform(-1, 1, (m, k)), rng.uniform(-1, 1, (k, n))
    c0 = rng.uniform(-1, 1, (m, n))
    got = oracle.gemm_f64(a, b, alpha=0.5, beta=2.0, c=c0)
    assert np.max(np.abs(got - (0.5 * (a @ b) + 2.0 * c0))) < 1e-13
    # k == 0: C = beta * C (outer.rs:213-229)
    z = oracle.gemm_f64(np.zeros((m, 0)), np.zeros((0, n)), beta=3.0, c=c0)
    assert np.array_equal(z, 3.0 * c0)


def test_normwise_sampling_consistent(oracle):
    rng = np.random.default_rng(5)
    m, n, k = 300, 280, 64
    a, b = rng.uniform(-1, 1, (m, k)), rng.uniform(-1, 1, (k, n))
    c = (a.astype(np.float32) @ b.astype(np.float32)).astype(np.float64)
    full = oracle.normwise_error(c, oracle.dd_full(a, b), m, n, oracle.fro(a), oracle.fro(b))
    sampled = oracle.error_vs_dd(a, b, c)
    assert 0.5 < sampled / full < 2.0


def test_half_restatements_widen_exactly(oracle):
    rng = np.random.default_rng(11)
    x = rng.standard_normal((7, 5)).astype(np.float32)
    bits = (x.view(np.uint32) >> 16).astype(np.uint16)      # truncate to bf16
    w = oracle.bf16_to_f32(bits)
    assert np.all((w.view(np.uint32) & 0xFFFF) == 0)
    assert np.all(np.abs(w - x) <= np.abs(x) * 2.0 ** -7)
    a16 = rng.standard_normal((6, 9)).astype(np.float16)
    b16 = rng.standard_normal((9, 4)).astype(np.float16)
    got = oracle.gemm_f16_f32(a16, b16)
    np.testing.assert_array_equal(got, oracle.gemm_f32(a16.astype(np.float32), b16.astype(np.float32)))
    c0 = rng.standard_normal((6, 4)).astype(np.float32)
    acc = oracle.gemm_f16_f32(a16, b16, c=c0.copy(), accumulate=True)
    np.testing.assert_array_equal(acc, oracle.gemm_f32(a16.astype(np.float32), b16.astype(np.float32),
                                                       1.0, 1.0, c0.copy()))


@pytest.mark.parametrize("case", __import__("trsm_cases").CASES, ids=lambda c: c[0])
def test_trsm_restatement_reference_cases(oracle, case):
    """The TRSM restatement passes the reference's own residual tests."""
    import trsm_cases as tc
    a, b = tc.operands(case)
    x = oracle.trsm_left(a, b, alpha=case[6], upper=case[2], unit_diag=case[3])
    assert x.dtype == b.dtype
    assert tc.residual_ok(case, a, b, x)


def test_trsm_restatement_unit_diag_and_empty(oracle):
    import trsm_cases as tc
    a = tc.unit_diag_triangle()
    b = (np.arange(24) * 0.3 + 0.5).reshape(6, 4)
    xu = oracle.trsm_left(a, b, unit_diag=True)
    xe = oracle.trsm_left(a, b, unit_diag=False)
    assert np.abs(xu - xe).max() < 1e-12
    e = np.zeros((0, 3))
    assert oracle.trsm_left(np.zeros((0, 0)), e).shape == (0, 3)


def test_trsm_restatement_split_rule(oracle):
    """m1 = min(round_up(m / 2, 32), m - 32): leaves for m = 100 are 64 -> (32, 32)
    and 36 -> (4, 32); the restatement's result is the same whatever the
    recursion (exact arithmetic), so check it against a dense solve."""
    import trsm_cases as tc
    for m in (33, 64, 100, 129):
        a = tc.random_triangle(m, np.float64, False, m)
        b = np.random.default_rng(m).standard_normal((m, 5))
        x = oracle.trsm_left(a, b)
        np.testing.assert_allclose(x, np.linalg.solve(a, b), rtol=1e-12, atol=1e-12)


def _pick_grid_py(m, n, k, workers, budget, mr=4):
    """outer.rs:343-383 (f64 budget 128 Ki, f32 256 Ki elements)."""
    import math
    if workers <= 1 or m == 0 or n == 0:
        return max(workers, 1), 1
    kc_eff = min(256, max(k, 1))
    chunks = m // mr
    if chunks >= workers and kc_eff * n <= budget:
        return workers, 1
    best, score_best = (1, workers), math.inf
    for mw in range(1, min(max(chunks, 1), workers) + 1):
        if workers % mw:
            continue
        nw = workers // mw
        sc = abs(math.log(m / mw) - math.log(n / nw))
        if sc < score_best or (sc == score_best and mw > best[0]):
            best, score_best = (mw, nw), sc
    return best


@pytest.mark.parametrize("m,n,k", [(8192, 8192, 8192), (160, 8192, 8192), (1024, 1024, 1024),
                                   (4096, 64, 300), (9, 5000, 40), (300, 300, 300), (32, 32, 32)])
def test_pick_grid_matches_reference_rule(oracle, m, n, k):
    for workers in (1, 3, 8):
        for f32 in (False, True):
            par, mw, nw = oracle.pick_grid(m, n, k, workers, f32)
            assert (mw, nw) == _pick_grid_py(m, n, k, workers, 256 * 1024 if f32 else 128 * 1024)
            assert par == (max(m, n, k) >= 256 and m >= 8)


def test_thread_grid_never_changes_a_bit(oracle):
    # 1-D slabs, 2-D cells and the sequential path agree bit for bit
    # (every element's chain is independent of the grid and of packing).
    rng = np.random.default_rng(12)
    for m, n, k in [(8, 4096, 300), (520, 600, 257), (64, 33, 700)]:
        a32, b32 = rng.standard_normal((m, k), dtype=np.float32), rng.standard_normal((k, n), dtype=np.float32)
        a64, b64 = a32.astype(np.float64), b32.astype(np.float64)
        ac = (a64 + 1j * a64[::-1]).astype(np.complex64)
        bc = (b64 - 1j * b64[::-1]).astype(np.complex64)
        a8, b8 = rng.integers(-128, 128, (m, k), dtype=np.int8), rng.integers(-128, 128, (k, n), dtype=np.int8)
        outs = []
        for th in (1, 3, 8):
            oracle.set_threads(th)
            outs.append((oracle.gemm_f32(a32, b32), oracle.gemm_f64(a64, b64), oracle.gemm_complex(ac, bc),
                         oracle.gemm_i8_signed(a8, b8)))
        oracle.set_threads(0)
        for o in outs[1:]:
            for x, y in zip(o, outs[0]):
                assert np.array_equal(x.view(np.uint8), y.view(np.uint8))
        np.testing.assert_array_equal(outs[0][3], oracle.gemm_i8_signed_rows(a8, b8))
