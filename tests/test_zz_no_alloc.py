"""fg_quantized_matmul_noalloc: the quantized GEMM for callers that may not
allocate device memory while they run (their memory belongs to another
allocator, or to a fixed budget).  Its row/column-sum scratch is a fixed
device array shared by every call, so the tests make calls in a row with
different operands -- a call that read the previous call's sums would
differ -- and check each one bit for bit against the oracle's restatement of
ferray's quantized_matmul and against fg_quantized_matmul, which takes its
scratch from the allocator.  Kept in its own file, collected last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(fg, lib, name, a, a_zp, sa, b, b_zp, sb, c0, accumulate):
    m, k = a.shape
    n = b.shape[1]
    ctx = fg.default_context()
    da, db, dc = fg.DeviceArray.from_numpy(a), fg.DeviceArray.from_numpy(b), fg.DeviceArray.from_numpy(c0)
    st = getattr(lib, name)(ctx.handle, m, n, k, da.ptr, a_zp, sa, db.ptr, b_zp, sb, dc.ptr,
                            int(accumulate), None)
    assert st == 0, lib.fg_last_error()
    ctx.sync()
    return dc.to_numpy()


def _case(rng, m, n, k):
    a = rng.integers(0, 256, (m, k), dtype=np.uint8)
    b = rng.integers(-128, 128, (k, n), dtype=np.int8)
    c0 = rng.standard_normal((m, n)).astype(np.float32)
    a_zp, b_zp = int(rng.integers(1, 256)), int(rng.integers(1, 128))  # both non-zero: every sum is read
    return a, b, c0, a_zp, b_zp


def test_noalloc_matches_oracle_and_allocating_entry_point_twice(fg, oracle):
    from ferray_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(2024)
    shapes = [(300, 272, 144, False), (129, 512, 1024, True)]  # k, n multiples of 16
    for m, n, k, accumulate in shapes:
        a, b, c0, a_zp, b_zp = _case(rng, m, n, k)
        sa, sb = np.float32(0.0123), np.float32(0.0456)
        want = oracle.quantized_matmul(a, a_zp, sa, b, b_zp, sb, c=c0.copy() if accumulate else None,
                                       accumulate=accumulate)
        alloc = _run(fg, lib, "fg_quantized_matmul", a, a_zp, sa, b, b_zp, sb, c0, accumulate)
        got = _run(fg, lib, "fg_quantized_matmul_noalloc", a, a_zp, sa, b, b_zp, sb, c0, accumulate)
        np.testing.assert_array_equal(got, want)
        np.testing.assert_array_equal(alloc, want)


def test_noalloc_many_rows_after_a_different_call(fg, oracle):
    """m = 40000 rows: more than one capped row-sum launch has warps, so every
    row's sum must be written by this call; the call before it left other
    sums in the shared array."""
    from ferray_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(77)
    m, n, k = 40000, 32, 48
    sa, sb = np.float32(0.5), np.float32(0.25)
    for _ in range(2):
        a, b, c0, a_zp, b_zp = _case(rng, m, n, k)
        got = _run(fg, lib, "fg_quantized_matmul_noalloc", a, a_zp, sa, b, b_zp, sb, c0, False)
        np.testing.assert_array_equal(got, oracle.quantized_matmul(a, a_zp, sa, b, b_zp, sb))


def test_noalloc_k_zero(fg):
    """k = 0 (gemm/mod.rs:509-519): C is zeroed, or left as it is when
    accumulating."""
    from ferray_b200 import _lib
    lib = _lib.load()
    ctx = fg.default_context()
    c0 = np.random.default_rng(5).standard_normal((40, 32)).astype(np.float32)
    for accumulate, want in ((True, c0), (False, np.zeros_like(c0))):
        dc = fg.DeviceArray.from_numpy(c0)
        st = lib.fg_quantized_matmul_noalloc(ctx.handle, 40, 32, 0, None, 3, 1.0, None, -2, 1.0, dc.ptr,
                                             int(accumulate), None)
        assert st == 0, lib.fg_last_error()
        ctx.sync()
        np.testing.assert_array_equal(dc.to_numpy(), want)


def test_noalloc_rejects_sizes_beyond_its_scratch(fg):
    from ferray_b200 import _lib
    lib = _lib.load()
    ctx = fg.default_context()
    st = lib.fg_quantized_matmul_noalloc(ctx.handle, 70000, 16, 16, C.c_void_p(16), 0, 1.0,
                                         C.c_void_p(16), 0, 1.0, C.c_void_p(16), 0, None)
    assert st == _lib.FG_ERR_UNSUPPORTED
    assert b"65536" in lib.fg_last_error()
