"""Served matmul stream measurement (used by bench.py).

Request mix of the served-stream config: 70% of requests with M, N, K
log-uniform in [16, 256], 25% in [256, 2048], 5% square 4096; dtypes 60% f32,
25% f64, 15% i8; Poisson arrivals at a given rate; 40 GB HBM budget.

Two arms on the same arrival stream:
* 'server': the continuous-batching server (split modes for floats: 3xBF16
  f32, Ozaki f64; small f32 / i8 requests folded into grouped launches,
  launches overlapped on several streams);
* 'plain': one call at a time in arrival order, plain mode, each synchronised
  before the next starts.
Latency = completion time - arrival time, per request.
"""
import ctypes as C
import queue as Q
import threading
import time

import numpy as np

SEED = 42


def workload(nreq, seed=SEED):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(nreq):
        u = rng.uniform()
        if u < 0.70:
            m, n, k = np.rint(np.exp(rng.uniform(np.log(16), np.log(256), 3))).astype(int)
        elif u < 0.95:
            m, n, k = np.rint(np.exp(rng.uniform(np.log(256), np.log(2048), 3))).astype(int)
        else:
            m = n = k = 4096
        v = rng.uniform()
        dt = np.float32 if v < 0.60 else (np.float64 if v < 0.85 else np.int8)
        out.append((int(m), int(n), int(k), dt))
    return out


def _fgdt(L, dt):
    return {np.dtype(np.float32): L.FG_F32, np.dtype(np.float64): L.FG_F64,
            np.dtype(np.int8): L.FG_I8}[np.dtype(dt)]


def run(fg, L, lib, ctx, reqs, rate, arm, pools, budget=40 << 30):
    """Offer `reqs` at Poisson rate `rate` (req/s) to one arm; returns a dict."""
    rng = np.random.default_rng(SEED + 7)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, len(reqs)))
    outs, off = [], 0
    for (m, n, k, dt) in reqs:
        es = 4 if dt == np.int8 else np.dtype(dt).itemsize
        outs.append(off)
        off += ((m * n * es + 255) // 256) * 256
    cbuf = fg.DeviceArray((max(off, 1),), np.uint8, ctx)
    done = [0.0] * len(reqs)
    flops = sum(2.0 * m * n * k for (m, n, k, _) in reqs)
    stats = None
    t0 = time.perf_counter() + 0.05
    if arm == "server":
        srv = fg.Server(hbm_budget_bytes=budget, streams=6, max_group=512, ctx=ctx)
        tickets = [None] * len(reqs)

        def waiter():
            for i in range(len(reqs)):
                while tickets[i] is None:
                    time.sleep(2e-5)
                srv.wait(tickets[i], timeout_ms=600000)
                done[i] = time.perf_counter()
        th = threading.Thread(target=waiter)
        th.start()
        for i, (m, n, k, dt) in enumerate(reqs):
            now = time.perf_counter()
            if t0 + arrivals[i] > now:
                time.sleep(t0 + arrivals[i] - now)
            a, b = pools[np.dtype(dt)]
            mode = L.FG_MODE_PLAIN if dt == np.int8 else L.FG_MODE_SPLIT
            req = L.fg_request(_fgdt(L, dt), mode, m, n, k, a.ptr, b.ptr, cbuf.ptr + outs[i], 0)
            t = C.c_uint64()
            st = lib.fg_server_submit(srv.handle, C.byref(req), C.byref(t))
            assert st == 0, lib.fg_last_error()
            tickets[i] = t.value
        th.join()
        stats = srv.stats()
        srv.stop()
    else:
        q = Q.Queue()

        def worker():
            one64, z64 = (C.c_double * 2)(1.0, 0.0), (C.c_double * 2)(0.0, 0.0)
            one32, z32 = (C.c_float * 2)(1.0, 0.0), (C.c_float * 2)(0.0, 0.0)
            while True:
                i = q.get()
                if i is None:
                    return
                m, n, k, dt = reqs[i]
                a, b = pools[np.dtype(dt)]
                f32 = dt == np.float32
                st = lib.fg_gemm(ctx.handle, _fgdt(L, dt), L.FG_MODE_PLAIN, 0, m, n, k,
                                 one32 if f32 else one64, a.ptr, k, b.ptr, n,
                                 z32 if f32 else z64, cbuf.ptr + outs[i], n, 0, None)
                assert st == 0, lib.fg_last_error()
                assert lib.fg_sync(ctx.handle, None) == 0
                done[i] = time.perf_counter()
        th = threading.Thread(target=worker)
        th.start()
        for i in range(len(reqs)):
            now = time.perf_counter()
            if t0 + arrivals[i] > now:
                time.sleep(t0 + arrivals[i] - now)
            q.put(i)
        q.put(None)
        th.join()
    lat = np.array([(done[i] - (t0 + arrivals[i])) * 1e3 for i in range(len(reqs))])
    span = max(done) - t0
    res = {"arm": arm, "rate_req_s": rate, "requests": len(reqs),
           "offered_s": round(float(arrivals[-1]), 3),
           "p50_ms": round(float(np.percentile(lat, 50)), 3),
           "p99_ms": round(float(np.percentile(lat, 99)), 3),
           "tflops": round(flops / span / 1e12, 2)}
    if stats:
        res["launches"] = int(stats["launches"])
        res["grouped_launches"] = int(stats["grouped_launches"])
        res["hbm_peak_gb"] = round(stats["hbm_peak"] / 1e9, 2)
    cbuf.free()
    return res


def sweep(fg, L, lib, ctx, rates, nreq):
    reqs = workload(nreq)
    rng = np.random.default_rng(3)
    big = 4096 * 4096
    pools = {
        np.dtype(np.float32): tuple(fg.DeviceArray.from_numpy(rng.standard_normal(big, dtype=np.float32), ctx)
                                    for _ in range(2)),
        np.dtype(np.float64): tuple(fg.DeviceArray.from_numpy(rng.standard_normal(big), ctx) for _ in range(2)),
        np.dtype(np.int8): tuple(fg.DeviceArray.from_numpy(rng.integers(-128, 128, big, dtype=np.int8), ctx)
                                 for _ in range(2)),
    }
    # warm both arms on the whole stream once (every tuned kernel variant the
    # stream reaches is loaded, attributes set, memory pools grown), so the
    # measured runs see a server in steady state
    run(fg, L, lib, ctx, reqs, max(rates), "server", pools)
    run(fg, L, lib, ctx, reqs, max(rates), "plain", pools)
    out = []
    for r in rates:
        out.append({"server": run(fg, L, lib, ctx, reqs, r, "server", pools),
                    "plain": run(fg, L, lib, ctx, reqs, r, "plain", pools)})
    return out
