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
