"""GPU tests of the continuous-batching server.

The required property: each result is the same whether its request ran alone
or in a concurrent mix (bit-identical: a request's kernel route depends only
on its class, never on what it is batched with), and every result meets the
parity tolerances against the oracle."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mix(fg, rng, count):
    reqs = []
    for i in range(count):
        kind = i % 6
        if kind in (0, 1):      # small f32, plain / split -> grouped
            m, n, k = rng.integers(16, 257, 3)
            a = rng.standard_normal((m, k)).astype(np.float32)
            b = rng.standard_normal((k, n)).astype(np.float32)
            mode = "plain" if kind == 0 else "split"
        elif kind == 2:         # small i8 -> grouped
            m, n, k = rng.integers(16, 257, 3)
            a = rng.integers(-128, 128, (m, k), dtype=np.int8)
            b = rng.integers(-128, 128, (k, n), dtype=np.int8)
            mode = "plain"
        elif kind == 3:         # f64 plain -> own launch
            m, n, k = rng.integers(16, 300, 3)
            a, b = rng.uniform(-1, 1, (m, k)), rng.uniform(-1, 1, (k, n))
            mode = "plain"
        elif kind == 4:         # f64 split (Ozaki) -> own launch
            m, n, k = rng.integers(16, 300, 3)
            a, b = rng.uniform(-1, 1, (m, k)), rng.uniform(-1, 1, (k, n))
            mode = "split"
        else:                   # larger f32 -> own launch
            m, n, k = 1100, 700, 1300
            a = rng.standard_normal((m, k)).astype(np.float32)
            b = rng.standard_normal((k, n)).astype(np.float32)
            mode = "split"
        out_dt = np.int32 if a.dtype == np.int8 else a.dtype
        reqs.append((fg.DeviceArray.from_numpy(a), fg.DeviceArray.from_numpy(b),
                     fg.DeviceArray((a.shape[0], b.shape[1]), out_dt), mode, a, b))
    return reqs


def test_server_results_same_alone_and_in_mix(fg, oracle):
    rng = np.random.default_rng(77)
    reqs = _mix(fg, rng, 48)
    srv = fg.Server(hbm_budget_bytes=8 << 30, streams=4, max_group=64)
    alone = []
    for da, db, dc, mode, a, b in reqs:
        srv.wait(srv.submit(da, db, dc, mode))
        alone.append(dc.to_numpy())
        fg.DeviceArray.from_numpy(np.zeros(dc.shape, dc.dtype))  # fresh buffers below
    # mix: clear outputs, submit everything from 4 threads at once
    for da, db, dc, *_ in reqs:
        z = np.zeros(dc.shape, dc.dtype)
        fg.default_context()._lib.fg_upload(fg.default_context().handle, dc.ptr, z.ctypes.data, z.nbytes, None)
    fg.default_context().sync()
    tickets = [None] * len(reqs)

    def worker(idx):
        for i in idx:
            da, db, dc, mode, *_ = reqs[i]
            tickets[i] = srv.submit(da, db, dc, mode)
    ths = [threading.Thread(target=worker, args=(range(t, len(reqs), 4),)) for t in range(4)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    for t in tickets:
        srv.wait(t, timeout_ms=60000)
    st = srv.stats()
    srv.stop()
    assert st["completed"] == 2 * len(reqs)
    assert st["grouped_launches"] >= 1
    assert st["p99_ms"] >= st["p50_ms"] > 0
    for (da, db, dc, mode, a, b), x in zip(reqs, alone):
        y = dc.to_numpy()
        np.testing.assert_array_equal(x, y)
        if a.dtype == np.int8:
            np.testing.assert_array_equal(y, (a.astype(np.int64) @ b.astype(np.int64)).astype(np.int32))
        else:
            k = a.shape[1]
            u = 2.0 ** -53 if a.dtype == np.float64 else 2.0 ** -24
            tol = k * u + (2.0 ** -15 if (mode == "split" and a.dtype == np.float32) else 0.0)
            assert oracle.error_vs_dd(a, b, y) <= tol


def test_server_budget(fg):
    rng = np.random.default_rng(5)
    a = fg.DeviceArray.from_numpy(rng.standard_normal((256, 256)).astype(np.float32))
    b = fg.DeviceArray.from_numpy(rng.standard_normal((256, 256)).astype(np.float32))
    cs = [fg.DeviceArray((256, 256), np.float32) for _ in range(8)]
    # room for about one request at a time: all still complete, in order
    srv = fg.Server(hbm_budget_bytes=1 << 20, streams=2)
    ts = [srv.submit(a, b, c) for c in cs]
    for t in ts:
        srv.wait(t, timeout_ms=60000)
    assert srv.stats()["hbm_peak"] <= 1 << 20
    big_a = fg.DeviceArray((2048, 2048), np.float32)
    big_c = fg.DeviceArray((2048, 2048), np.float32)
    with pytest.raises(fg.BudgetExceeded):
        srv.submit(big_a, big_a, big_c)
    srv.stop()
    want = a.to_numpy() @ b.to_numpy()
    for c in cs:
        assert np.max(np.abs(c.to_numpy() - want)) < 1e-3
