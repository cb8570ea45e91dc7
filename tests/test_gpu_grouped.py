"""GPU tests of the grouped (ragged-batch) GEMM: one persistent launch over a
device problem table, one-shot and replayed from a CUDA graph plan.

i8 problems must be bit-exact (wrapping int32); f32 problems must meet the
normwise tolerances of test_gpu_parity (plain FFMA: K * 2^-24; split 3xBF16:
2^-15 + K * 2^-24) against the double-double oracle, problem by problem.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

U32 = 2.0 ** -24


def ragged_dims(rng, count, lo=8, hi=512):
    return np.rint(np.exp(rng.uniform(np.log(lo), np.log(hi), (count, 3)))).astype(int)


def make_problems(fg, rng, dims, dtype):
    probs, host = [], []
    for m, n, k in dims:
        if dtype == np.int8:
            a = rng.integers(-128, 128, (m, k), dtype=np.int8)
            b = rng.integers(-128, 128, (k, n), dtype=np.int8)
            c = np.zeros((m, n), np.int32)
        else:
            a = rng.standard_normal((m, k)).astype(np.float32)
            b = rng.standard_normal((k, n)).astype(np.float32)
            c = np.zeros((m, n), np.float32)
        da, db, dc = (fg.DeviceArray.from_numpy(x) for x in (a, b, c))
        probs.append((m, n, k, da, db, dc))
        host.append((a, b))
    return probs, host


def check(fg, oracle, probs, host, dtype, mode):
    for (m, n, k, da, db, dc), (a, b) in zip(probs, host):
        got = dc.to_numpy()
        if dtype == np.int8:
            want = (a.astype(np.int64) @ b.astype(np.int64)).astype(np.int32)
            np.testing.assert_array_equal(got, want)
        else:
            err = oracle.error_vs_dd(a, b, got)
            tol = k * U32 if mode == "plain" else 2.0 ** -15 + k * U32
            assert err <= tol, (m, n, k, err)


@pytest.mark.parametrize("dtype,mode", [(np.int8, "plain"), (np.float32, "plain"),
                                        (np.float32, "split")])
def test_grouped_one_shot(fg, oracle, dtype, mode):
    rng = np.random.default_rng(11)
    dims = ragged_dims(rng, 48)
    dims = np.vstack([dims, [[1, 1, 1], [3, 700, 5], [600, 2, 17], [129, 257, 300]]])
    probs, host = make_problems(fg, rng, dims, dtype)
    fg.gemm_grouped(probs, dtype=dtype, mode=mode)
    check(fg, oracle, probs, host, dtype, mode)


@pytest.mark.parametrize("dtype,mode", [(np.int8, "plain"), (np.float32, "split"), (np.float32, "plain")])
def test_grouped_plan_replay(fg, oracle, dtype, mode):
    rng = np.random.default_rng(12)
    dims = ragged_dims(rng, 64)
    probs, host = make_problems(fg, rng, dims, dtype)
    plan = fg.GroupedPlan(probs, dtype=dtype, mode=mode)
    plan.run()
    check(fg, oracle, probs, host, dtype, mode)
    # new operand values, same buffers: a replay must pick them up
    host2 = []
    for (m, n, k, da, db, dc), (a, b) in zip(probs, host):
        a2 = (a[::-1].copy() if dtype == np.int8 else (a * 0.5).astype(np.float32))
        da_h = np.ascontiguousarray(a2)
        fg.default_context()._lib.fg_upload(fg.default_context().handle, da.ptr, da_h.ctypes.data,
                                            da_h.nbytes, None)
        host2.append((da_h, b))
    fg.default_context().sync()
    plan.run()
    check(fg, oracle, probs, host2, dtype, mode)
    plan.close()


def test_grouped_k_zero_and_empty(fg):
    rng = np.random.default_rng(13)
    a = fg.DeviceArray.from_numpy(np.zeros((5, 0), np.float32))
    b = fg.DeviceArray.from_numpy(np.zeros((0, 7), np.float32))
    c = fg.DeviceArray.from_numpy(rng.standard_normal((5, 7)).astype(np.float32))
    a2 = fg.DeviceArray.from_numpy(rng.standard_normal((4, 9)).astype(np.float32))
    b2 = fg.DeviceArray.from_numpy(rng.standard_normal((9, 6)).astype(np.float32))
    c2 = fg.DeviceArray((4, 6), np.float32)
    fg.gemm_grouped([(5, 7, 0, a, b, c), (4, 6, 9, a2, b2, c2)], dtype=np.float32)
    assert np.all(c.to_numpy() == 0.0)
    assert np.max(np.abs(c2.to_numpy() - a2.to_numpy() @ b2.to_numpy())) < 1e-4
    fg.gemm_grouped([], dtype=np.float32)


def _placed(rng, dims, esize, aligned_every=4):
    """Operand placements inside one device buffer: per problem a byte offset
    and leading dimensions.  Every `aligned_every`-th problem gets 16-byte
    offsets and leading dimensions (TMA reads it); the others get odd offsets
    and padded leading dimensions (the prep pass re-pitches those)."""
    out, cur = [], 0
    for i, (m, n, k) in enumerate(dims):
        if i % aligned_every == 0:
            k16, n16 = -(-k // 16) * 16, -(-n // 16) * 16
            lda, ldb = k16 + 16 * int(rng.integers(0, 2)), n16 + 16 * int(rng.integers(0, 2))
            oa = -(-cur // 16) * 16
        else:
            lda, ldb = k + int(rng.integers(0, 5)), n + int(rng.integers(0, 5))
            oa = cur + int(rng.integers(1, 16)) * (1 if esize == 1 else 0) + esize * int(rng.integers(1, 4))
        ob = oa + esize * m * lda
        ob = -(-ob // 16) * 16 + (0 if i % aligned_every == 0 else esize * int(rng.integers(1, 4)))
        cur = ob + esize * k * ldb + 64
        out.append((oa, ob, lda, ldb))
    return out, cur


@pytest.mark.parametrize("dtype", [np.int8, np.uint8])
def test_grouped_i8_offsets_and_padding(fg, dtype):
    """i8 / u8 x i8 problems at unaligned offsets with padded leading
    dimensions (re-pitched by the prep pass), mixed in one launch with 16-byte-aligned ones
    (TMA), padded output rows too: bit-exact against int64 products."""
    rng = np.random.default_rng(21)
    dims = ragged_dims(rng, 40, 1, 300)
    dims = np.vstack([dims, [[1, 1, 1], [130, 3, 260], [5, 129, 17], [256, 256, 256]]])
    place, total = _placed(rng, dims, 1)
    buf = np.full(total, 0x5A, np.uint8)  # padding bytes must not leak into results
    want, outs = [], []
    for (m, n, k), (oa, ob, lda, ldb) in zip(dims, place):
        a = rng.integers(0, 256, (m, k), dtype=np.uint8)
        b = rng.integers(0, 256, (k, n), dtype=np.uint8)
        for r in range(m):
            buf[oa + r * lda: oa + r * lda + k] = a[r]
        for r in range(k):
            buf[ob + r * ldb: ob + r * ldb + n] = b[r]
        av = a.astype(np.int64) if dtype == np.uint8 else a.view(np.int8).astype(np.int64)
        want.append((av @ b.view(np.int8).astype(np.int64)).astype(np.int32))
    dbuf = fg.DeviceArray.from_numpy(buf)
    probs = []
    for (m, n, k), (oa, ob, lda, ldb) in zip(dims, place):
        ldc = n + int(rng.integers(0, 3))
        dc = fg.DeviceArray.from_numpy(np.full((m, ldc), -7, np.int32))
        outs.append((dc, n))
        probs.append((int(m), int(n), int(k), dbuf.ptr + oa, dbuf.ptr + ob, dc.ptr, lda, ldb, ldc))
    fg.gemm_grouped(probs, dtype=dtype)
    for (dc, n), w in zip(outs, want):
        got = dc.to_numpy()
        np.testing.assert_array_equal(got[:, :n], w)
        assert np.all(got[:, n:] == -7), "store past the row end"


def test_grouped_split_offsets_and_padding(fg, oracle):
    """Split-f32 problems whose operands sit at 4-byte (not 16-byte) offsets
    with padded leading dimensions: within tolerance of the DD oracle, and
    bit-identical to the same problems from contiguous buffers (the split
    pass reads both, so placement must not change a bit)."""
    rng = np.random.default_rng(22)
    dims = ragged_dims(rng, 24, 1, 300)
    dims = np.vstack([dims, [[1, 1, 1], [130, 3, 260], [5, 129, 17]]])
    place, total = _placed(rng, dims, 4, aligned_every=3)
    buf = np.full(total // 4 + 16, np.nan, np.float32)  # padding must not leak
    host, probs, probs_c, outs = [], [], [], []
    for (m, n, k), (oa, ob, lda, ldb) in zip(dims, place):
        a = rng.standard_normal((m, k)).astype(np.float32)
        b = rng.standard_normal((k, n)).astype(np.float32)
        for r in range(m):
            buf[oa // 4 + r * lda: oa // 4 + r * lda + k] = a[r]
        for r in range(k):
            buf[ob // 4 + r * ldb: ob // 4 + r * ldb + n] = b[r]
        host.append((a, b))
    dbuf = fg.DeviceArray.from_numpy(buf)
    keep = []
    for (m, n, k), (oa, ob, lda, ldb), (a, b) in zip(dims, place, host):
        dc = fg.DeviceArray((m, n), np.float32)
        probs.append((int(m), int(n), int(k), dbuf.ptr + oa, dbuf.ptr + ob, dc.ptr, lda, ldb, int(n)))
        da, db = fg.DeviceArray.from_numpy(a), fg.DeviceArray.from_numpy(b)
        dc2 = fg.DeviceArray((m, n), np.float32)
        keep += [da, db]
        probs_c.append((int(m), int(n), int(k), da, db, dc2))
        outs.append((dc, dc2))
    fg.gemm_grouped(probs, dtype=np.float32, mode="split")
    fg.gemm_grouped(probs_c, dtype=np.float32, mode="split")
    for (m, n, k), (dc, dc2), (a, b) in zip(dims, outs, host):
        got = dc.to_numpy()
        assert np.array_equal(got.view(np.uint32), dc2.to_numpy().view(np.uint32)), (m, n, k)
        err = oracle.error_vs_dd(a, b, got)
        assert err <= 2.0 ** -15 + k * U32, (m, n, k, err)


@pytest.mark.parametrize("dtype,mode", [(np.int8, "plain"), (np.float32, "split")])
def test_grouped_row_spread_boundaries(fg, oracle, dtype, mode):
    """Tile heights at every boundary of the kernels' row spreading (A rows
    loaded as 8-row boxes spread over the four accumulator lane quadrants,
    each epilogue warp storing rows 8 w + 32 j + r): M around 8, 32, 64, 96,
    128 and past one tile, with ragged N and K.  i8 exact; split f32 within
    the DD tolerance; rows of C outside the product are left alone."""
    rng = np.random.default_rng(23)
    ms = [1, 7, 8, 9, 31, 32, 33, 63, 64, 65, 96, 97, 127, 128, 129, 255, 257]
    dims = np.array([[m, int(rng.integers(1, 200)), int(rng.integers(1, 300))] for m in ms])
    probs, host = make_problems(fg, rng, dims, dtype)
    # C one row taller than the product, guard row filled: the extra row must survive
    guarded = []
    for (m, n, k, da, db, dc) in probs:
        fill = np.full((m + 1, n), -9 if dtype == np.int8 else np.float32(-9.5),
                       np.int32 if dtype == np.int8 else np.float32)
        g = fg.DeviceArray.from_numpy(fill)
        guarded.append((m, n, k, da, db, g))
    fg.gemm_grouped(guarded, dtype=dtype, mode=mode)
    for (m, n, k, da, db, g), (a, b) in zip(guarded, host):
        got = g.to_numpy()
        assert np.all(got[m] == (-9 if dtype == np.int8 else np.float32(-9.5))), (m, n, k)
        got = got[:m]
        if dtype == np.int8:
            want = (a.astype(np.int64) @ b.astype(np.int64)).astype(np.int32)
            np.testing.assert_array_equal(got, want)
        else:
            err = oracle.error_vs_dd(a, b, got)
            assert err <= 2.0 ** -15 + k * U32, (m, n, k, err)
