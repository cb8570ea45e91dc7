"""Failure detection on the device without a fault: a bounded wait that
nothing satisfies gives up, the host reads FG_ERR_TIMEOUT from fg_sync, and
the context keeps working (the next GEMM is exact, the next sync is OK)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_context_survives(fg, oracle):
    from ferray_b200 import _lib as L
    ctx = fg.default_context()
    lib = ctx._lib
    assert lib.fg_sync(ctx.handle, None) == L.FG_OK
    assert lib.fg_selftest_wait_timeout(ctx.handle, 2000, None) == L.FG_OK
    assert lib.fg_sync(ctx.handle, None) == L.FG_ERR_TIMEOUT
    assert b"site 127" in lib.fg_last_error()
    # the error word is cleared once reported; the device is still usable
    assert lib.fg_sync(ctx.handle, None) == L.FG_OK
    r = np.random.default_rng(0)
    a = r.integers(-128, 128, (64, 96), dtype=np.int8)
    b = r.integers(-128, 128, (96, 80), dtype=np.int8)
    c = np.zeros((64, 80), np.int32)
    assert fg.gemm_i8_signed(64, 80, 96, a, b, c)
    np.testing.assert_array_equal(c, oracle.gemm_i8_signed(a, b))
    assert lib.fg_sync(ctx.handle, None) == L.FG_OK


def test_selftest_rejects_unbounded_timeouts(fg):
    from ferray_b200 import _lib as L
    ctx = fg.default_context()
    assert ctx._lib.fg_selftest_wait_timeout(ctx.handle, 0, None) == L.FG_ERR_INVALID
    assert ctx._lib.fg_selftest_wait_timeout(ctx.handle, 2000000, None) == L.FG_ERR_INVALID

