"""fg_quantized_matmul_noalloc: the quantized GEMM for callers that may not
allocate device memory while they run (their memory belongs to another
allocator, or to a fixed budget).  Its row/column-sum scratch is a fixed
device array shared by every call, so the test makes two calls in a row with
different operands -- a second call that read the first call's sums would
differ -- and compares each, bit for bit, with fg_quantized_matmul, which
takes its scratch from the allocator.  Kept in its own file, collected last.
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


def test_noalloc_matches_allocating_entry_point_twice(fg):
    from ferray_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(2024)
    shapes = [(300, 272, 144, False), (129, 512, 1024, True)]  # k, n multiples of 16
    for m, n, k, accumulate in shapes:
        a = rng.integers(0, 256, (m, k), dtype=np.uint8)
        b = rng.integers(-128, 128, (k, n), dtype=np.int8)
        c0 = rng.standard_normal((m, n)).astype(np.float32)
        a_zp, b_zp = int(rng.integers(0, 256)), int(rng.integers(-128, 128))
        sa, sb = np.float32(0.0123), np.float32(0.0456)
        want = _run(fg, lib, "fg_quantized_matmul", a, a_zp, sa, b, b_zp, sb, c0, accumulate)
        got = _run(fg, lib, "fg_quantized_matmul_noalloc", a, a_zp, sa, b, b_zp, sb, c0, accumulate)
        np.testing.assert_array_equal(got, want)


def test_noalloc_rejects_sizes_beyond_its_scratch(fg):
    from ferray_b200 import _lib
    lib = _lib.load()
    ctx = fg.default_context()
    st = lib.fg_quantized_matmul_noalloc(ctx.handle, 70000, 16, 16, C.c_void_p(16), 0, 1.0,
                                         C.c_void_p(16), 0, 1.0, C.c_void_p(16), 0, None)
    assert st == _lib.FG_ERR_UNSUPPORTED
    assert b"65536" in lib.fg_last_error()
