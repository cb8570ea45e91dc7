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
Latency = completion time - scheduled arrival time, per request.  The server
arm takes each request's completion time from the server itself
(fg_server_wait_times: when its work was seen complete on the GPU), so the
order in which the host waits does not matter.

Operands: every request reads its own A and B, carved in turn from a
per-dtype device arena of 512 MiB (four times the 126 MB L2) filled with the
config's value distributions, so consecutive requests do not find their
operands in L2; every request writes its own C.
"""
import ctypes as C
import queue as Q
import threading
import time

import numpy as np

SEED = 42
ARENA_BYTES = 512 << 20


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


class Arenas:
    """Per-dtype operand arenas on the device and one output buffer."""

    def __init__(self, torch, reqs):
        gen = torch.Generator(device="cuda")
        gen.manual_seed(SEED)
        self.arena = {
            np.dtype(np.float32): torch.randn(ARENA_BYTES // 4, device="cuda", generator=gen),
            np.dtype(np.float64): torch.randn(ARENA_BYTES // 8, dtype=torch.float64, device="cuda",
                                              generator=gen),
            np.dtype(np.int8): torch.randint(-128, 128, (ARENA_BYTES,), dtype=torch.int8, device="cuda",
                                             generator=gen),
        }
        cursor = {d: 0 for d in self.arena}
        self.ab, self.c_off = [], []
        off = 0
        for (m, n, k, dt) in reqs:
            d = np.dtype(dt)
            es = d.itemsize
            base = self.arena[d].data_ptr()
            ptrs = []
            for elems in (m * k, k * n):
                nb = (elems * es + 255) // 256 * 256
                if cursor[d] + nb > ARENA_BYTES:
                    cursor[d] = 0
                ptrs.append(base + cursor[d])
                cursor[d] += nb
            self.ab.append(tuple(ptrs))
            self.c_off.append(off)
            off += ((m * n * (4 if dt == np.int8 else es) + 255) // 256) * 256
        self.c = torch.empty(max(off, 1), dtype=torch.uint8, device="cuda")


def run(fg, L, lib, ctx, reqs, rate, arm, arenas, budget=40 << 30):
    """Offer `reqs` at Poisson rate `rate` (req/s) to one arm; returns a dict."""
    rng = np.random.default_rng(SEED + 7)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, len(reqs)))
    cbase = arenas.c.data_ptr()
    done = [0.0] * len(reqs)
    flops = sum(2.0 * m * n * k for (m, n, k, _) in reqs)
    stats = None
    lag = 0.0
    if arm == "server":
        srv = fg.Server(hbm_budget_bytes=budget, streams=6, max_group=512, ctx=ctx)
        built = []
        for i, (m, n, k, dt) in enumerate(reqs):
            mode = L.FG_MODE_PLAIN if dt == np.int8 else L.FG_MODE_SPLIT
            a, b = arenas.ab[i]
            built.append(L.fg_request(_fgdt(L, dt), mode, m, n, k, a, b, cbase + arenas.c_off[i], 0))
        tickets = [None] * len(reqs)

        def waiter():
            for i in range(len(reqs)):
                while tickets[i] is None:
                    time.sleep(2e-5)
                _, done[i] = srv.wait_times(tickets[i], timeout_ms=600000)
        th = threading.Thread(target=waiter)
        th.start()
        p0, c0 = time.perf_counter(), srv.clock()
        t0 = p0 + 0.05
        t0_lib = c0 + 0.05
        t = C.c_uint64()
        submit = lib.fg_server_submit
        for i, req in enumerate(built):
            now = time.perf_counter()
            if t0 + arrivals[i] > now:
                time.sleep(t0 + arrivals[i] - now)
            else:
                lag = max(lag, now - (t0 + arrivals[i]))
            st = submit(srv.handle, C.byref(req), C.byref(t))
            assert st == 0, lib.fg_last_error()
            tickets[i] = t.value
        th.join()
        stats = srv.stats()
        srv.stop()
        lat = np.array([(done[i] - (t0_lib + arrivals[i])) * 1e3 for i in range(len(reqs))])
        span = max(done) - t0_lib
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
                a, b = arenas.ab[i]
                f32 = dt == np.float32
                st = lib.fg_gemm(ctx.handle, _fgdt(L, dt), L.FG_MODE_PLAIN, 0, m, n, k,
                                 one32 if f32 else one64, a, k, b, n,
                                 z32 if f32 else z64, cbase + arenas.c_off[i], n, 0, None)
                assert st == 0, lib.fg_last_error()
                assert lib.fg_sync(ctx.handle, None) == 0
                done[i] = time.perf_counter()
        th = threading.Thread(target=worker)
        th.start()
        t0 = time.perf_counter() + 0.05
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
        res["max_submit_lag_ms"] = round(lag * 1e3, 3)
    return res


def sweep(fg, L, lib, ctx, rates, nreq, seconds_per_rate=3.0):
    """Both arms at every rate; the request count at a rate is
    min(nreq, rate * seconds_per_rate) (at least 1000), the first requests of
    one seeded stream."""
    import torch
    counts = [int(min(nreq, max(1000, r * seconds_per_rate))) for r in rates]
    reqs = workload(max(counts))
    arenas = Arenas(torch, reqs)
    # warm both arms once (every tuned kernel variant the stream reaches is
    # loaded, attributes set, memory pools grown), so the measured runs see a
    # server in steady state
    warm = reqs[:min(len(reqs), 2000)]
    run(fg, L, lib, ctx, warm, max(rates), "server", arenas)
    run(fg, L, lib, ctx, warm, max(rates), "plain", arenas)
    out = []
    for r, cnt in zip(rates, counts):
        out.append({"server": run(fg, L, lib, ctx, reqs[:cnt], r, "server", arenas),
                    "plain": run(fg, L, lib, ctx, reqs[:cnt], r, "plain", arenas)})
    del arenas
    torch.cuda.empty_cache()
    return out
