"""Device TRSM (fg_trsm_left) against the restated reference
(ferray-linalg/src/trsm.rs): solves of up to 128 rows bit-identical, larger
ones within a normwise tolerance (their trailing GEMMs sum in another
order), and the reference's own residual tests."""
import numpy as np
import pytest

import trsm_cases as tc

pytestmark = pytest.mark.gpu

FUNCS = {(np.float64, False): "trsm_left_lower_f64", (np.float64, True): "trsm_left_upper_f64",
         (np.float32, False): "trsm_left_lower_f32", (np.float32, True): "trsm_left_upper_f32"}


def solve(fg, a, b, alpha=1.0, upper=False, unit=False, mode="plain", lda=None, ldb=None):
    dt = b.dtype.type
    m, n = b.shape
    lda, ldb = lda or m, ldb or n
    ap = np.zeros((m, lda), dt)
    ap[:, :m] = a
    bp = np.full((m, ldb), 7.0, dt)
    bp[:, :n] = b
    getattr(fg, FUNCS[(dt, upper)])(m, n, alpha, ap, lda, bp, ldb, unit, mode=mode)
    assert np.all(bp[:, n:] == 7.0), "columns past n were written"
    return bp[:, :n]


@pytest.mark.parametrize("case", tc.CASES, ids=lambda c: c[0])
def test_reference_cases(fg, oracle, case):
    a, b = tc.operands(case)
    x = solve(fg, a, b, alpha=case[6], upper=case[2], unit=case[3])
    assert tc.residual_ok(case, a, b, x)
    ref = oracle.trsm_left(a, b, alpha=case[6], upper=case[2], unit_diag=case[3])
    if case[4] <= 128:
        np.testing.assert_array_equal(x, ref)  # one block: the reference's exact operations
    else:
        tol = 1e-13 if b.dtype == np.float64 else 1e-5
        assert np.linalg.norm(x - ref) <= tol * np.linalg.norm(ref)


def test_unit_diag(fg):
    a = tc.unit_diag_triangle()
    b = (np.arange(24) * 0.3 + 0.5).reshape(6, 4)
    xu = solve(fg, a, b, unit=True)
    xe = solve(fg, a, b, unit=False)
    assert np.abs(xu - xe).max() < 1e-12


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("upper", [False, True])
@pytest.mark.parametrize("unit", [False, True])
@pytest.mark.parametrize("m,n", [(1, 1), (7, 129), (31, 1000), (32, 257), (33, 40), (65, 3), (100, 77),
                                 (127, 300), (128, 64)])
def test_block_bit_exact(fg, oracle, dt, upper, unit, m, n):
    a = tc.random_triangle(m, dt, upper, m + n)
    b = np.random.default_rng(n).standard_normal((m, n)).astype(dt)
    for alpha in (1.0, 2.5):
        x = solve(fg, a, b, alpha=alpha, upper=upper, unit=unit, lda=m + 3, ldb=n + 5)
        np.testing.assert_array_equal(x, oracle.trsm_left(a, b, alpha=alpha, upper=upper, unit_diag=unit))


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("upper", [False, True])
@pytest.mark.parametrize("mode", ["plain", "split"])
@pytest.mark.parametrize("m,n", [(129, 40), (300, 50), (1000, 777)])
def test_blocked_vs_restatement(fg, oracle, dt, upper, mode, m, n):
    a = tc.random_triangle(m, dt, upper, m * 7 + n)
    b = np.random.default_rng(m).standard_normal((m, n)).astype(dt)
    x = solve(fg, a, b, alpha=0.75, upper=upper, mode=mode, lda=m + 1, ldb=n + 2)
    ref = oracle.trsm_left(a, b, alpha=0.75, upper=upper)
    # normwise, relative to the solution: the trailing GEMMs round
    # differently from the reference's scalar loop (FMA, another order)
    tol = 1e-13 if dt == np.float64 else 4e-6
    assert np.linalg.norm(x.astype(np.float64) - ref) <= tol * np.linalg.norm(ref)


def test_device_in_place_and_empty(fg, oracle):
    m, n = 200, 64
    a = tc.random_triangle(m, np.float64, False, 5)
    b = np.random.default_rng(5).standard_normal((m, n))
    da, db = fg.DeviceArray.from_numpy(a), fg.DeviceArray.from_numpy(b)
    fg.trsm_left_lower_f64(m, n, 1.0, da, m, db, n, False)
    ref = oracle.trsm_left(a, b)
    assert np.linalg.norm(db.to_numpy() - ref) <= 1e-13 * np.linalg.norm(ref)
    e = np.zeros((0, 4))
    fg.trsm_left_lower_f64(0, 4, 2.0, np.zeros((0, 0)), 0, e, 4, False)  # no-op, as trsm.rs:56


def test_errors(fg):
    import ctypes as C
    from ferray_b200 import _lib as L
    ctx = fg.default_context()
    one = C.c_double(1.0)
    a = fg.DeviceArray.from_numpy(np.eye(4))
    b = fg.DeviceArray.from_numpy(np.ones((4, 4)))
    lib = ctx._lib
    assert lib.fg_trsm_left(ctx.handle, L.FG_I8, 0, 0, 0, 4, 4, C.byref(one), a.ptr, 4, b.ptr, 4,
                            None) == L.FG_ERR_DTYPE
    assert lib.fg_trsm_left(ctx.handle, L.FG_F64, 0, 0, 0, 4, 4, C.byref(one), a.ptr, 3, b.ptr, 4,
                            None) == L.FG_ERR_SHAPE
    assert lib.fg_trsm_left(ctx.handle, L.FG_F64, 0, 0, 0, 4, 4, C.byref(one), None, 4, b.ptr, 4,
                            None) == L.FG_ERR_INVALID
    with pytest.raises(fg.ShapeMismatch):
        fg.trsm_left_lower_f64(4, 4, 1.0, np.eye(4), 3, np.ones((4, 4)), 4, False)
