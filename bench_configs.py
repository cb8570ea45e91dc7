"""The benchmark configurations beside the headline SGEMM step, one function
each, every GPU number next to its error against the double-double oracle
and the CPU rate of ferray's restated GEMM (the oracle) on the same shape:

* DGEMM f64 M = N = K = 1024, U[-1, 1), plain and Ozaki split (scheme II
  with 16 moduli, the default, and scheme I with 9 slices), error vs the DD
  oracle over the full C;
* SGEMM f32 N in {256, 1024, 2048, 4096}, N(0, 1): plain FFMA, 3 x BF16
  (2 slices) and 6 x BF16 (3 slices) split;
* CGEMM c32 N = 4096, Re and Im N(0, 1): plain, 3- and 6-product split;
* DGEMM f64 / ZGEMM c128 at N in {2048, 4096, 8192} with exponent spread
  s in {0, 4, 8} (A = diag(10^(s u)) G diag(10^(s v)), G ~ N(0, 1),
  u, v ~ U[-1, 1]; B built the same way independently): plain FP64 vs
  INT8-Ozaki scheme I (8, 9 slices) and scheme II (16, 17 moduli), errors
  per spread;
* square i8 x i8 -> i32 at N in {1024, 4096, 8192}, bit-exact on a sample.

Workloads are seeded synthetic data with the configs' shapes and value
distributions.  GPU times are CUDA events on the launching stream over
back-to-back calls after warm-up; the CPU rates time the oracle on the
first rows of the same problem (all of it where it fits the time budget) on
ferray's pool of min(cores, 8) threads.
"""
import ctypes as C
import time

import numpy as np

SEED = 42


def pool_threads():
    """min(available parallelism, 8): ferray's GEMM pool
    (ferray-linalg/src/gemm/outer.rs:142-155)."""
    import os
    try:
        cores = len(os.sched_getaffinity(0))
    except AttributeError:
        cores = os.cpu_count() or 1
    return max(1, min(cores, 8))


# ----------------------------------------------------------------- CPU rates

def _cpu_operands(kind, rows, n, k, rng):
    if kind in ("f64", "f32"):
        dt = np.float64 if kind == "f64" else np.float32
        return rng.standard_normal((rows, k)).astype(dt), rng.standard_normal((k, n)).astype(dt)
    if kind in ("c128", "c64"):
        dt = np.complex128 if kind == "c128" else np.complex64
        a = (rng.standard_normal((rows, k)) + 1j * rng.standard_normal((rows, k))).astype(dt)
        b = (rng.standard_normal((k, n)) + 1j * rng.standard_normal((k, n))).astype(dt)
        return a, b
    return (rng.integers(-128, 128, (rows, k), dtype=np.int8),
            rng.integers(-128, 128, (k, n), dtype=np.int8))


def _cpu_call(oracle, kind):
    if kind == "f64":
        return oracle.gemm_f64
    if kind == "f32":
        return oracle.gemm_f32
    if kind in ("c128", "c64"):
        return oracle.gemm_complex
    return oracle.gemm_i8_signed


def cpu_rate(kind, m, n, k, budget_s=2.0, seed=SEED):
    """ferray's CPU GEMM (the oracle's restatement) on an m x n x k problem of
    dtype `kind` (f64, f32, c128, c64, i8): the first `rows` rows of C, all m
    when they fit `budget_s`, at least min(m, 64) (ferray's grid then splits
    N, so every pool thread still has work).  Rate in TFLOP/s (TOPS for i8),
    2mnk real / 8mnk complex."""
    import oracle
    threads = pool_threads()
    oracle.set_threads(threads)
    rng = np.random.default_rng(seed)
    fn = _cpu_call(oracle, kind)
    r0 = min(m, 64)
    a, b = _cpu_operands(kind, r0, n, k, rng)
    fn(a[:min(r0, 8)], b)  # warm the pack buffers
    t0 = time.perf_counter()
    fn(a, b)
    t = time.perf_counter() - t0
    rows = r0
    if rows < m and t < budget_s / 2:
        rows = min(m, max(r0, int(budget_s / (t / r0)) // 64 * 64))
        if rows > r0:
            a, _ = _cpu_operands(kind, rows, n, k, rng)
            t0 = time.perf_counter()
            fn(a, b)
            t = time.perf_counter() - t0
    if rows == m and t < budget_s / 4:  # small problems: median of repeats
        reps = max(3, min(30, int(budget_s / 2 / max(t, 1e-6))))
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            fn(a, b)
            ts.append(time.perf_counter() - t0)
        t = float(np.median(ts))
    flops = (8.0 if kind in ("c128", "c64") else 2.0) * rows * n * k
    return {"value": round(flops / t / 1e12, 4), "unit": "TOPS" if kind == "i8" else "TFLOP/s",
            "cores": threads, "kind": "port",
            "sample": ("all %d rows" % m if rows == m else "%d of %d rows of C" % (rows, m)) +
                      ", %.3f s per call" % t}


# ------------------------------------------------------------------ helpers

class Runner:
    """Calls through the C ABI on one stream, timed with CUDA events."""

    def __init__(self, fg, L, lib, ctx, stream):
        import torch
        self.torch, self.fg, self.L, self.lib, self.ctx, self.stream = torch, fg, L, lib, ctx, stream
        self.sh = C.c_void_p(stream.cuda_stream)

    def gemm(self, dtype, mode, slices, m, n, k, a, b, c):
        L = self.L
        if dtype in (L.FG_F64, L.FG_C64):
            al, be = (C.c_double * 2)(1.0, 0.0), (C.c_double * 2)(0.0, 0.0)
        else:
            al, be = (C.c_float * 2)(1.0, 0.0), (C.c_float * 2)(0.0, 0.0)

        def call():
            st = self.lib.fg_gemm(self.ctx.handle, dtype, mode, slices, m, n, k, al, a, k, b, n, be, c, n, 0,
                                  self.sh)
            if st != 0:
                raise RuntimeError(self.lib.fg_last_error().decode())
        return call

    def time(self, fn, min_ms=30.0, max_iters=200):
        torch = self.torch
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(self.stream)
        fn()
        e1.record(self.stream)
        torch.cuda.synchronize()
        one = max(e0.elapsed_time(e1), 1e-3)
        iters = int(max(2, min(max_iters, min_ms / one)))
        for _ in range(2):
            fn()
        e0.record(self.stream)
        for _ in range(iters):
            fn()
        e1.record(self.stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / iters


def _err(oracle, got_block, a_rows, b_cols, m, n, na, nb):
    ref = oracle.dd_sampled(a_rows, b_cols, np.arange(a_rows.shape[0]), np.arange(b_cols.shape[1]))
    return oracle.normwise_error(got_block, ref, m, n, na, nb)


def _entry(flops, ms, err=None, **kw):
    d = {"tflops": round(flops / ms / 1e9, 2), "ms": round(ms, 4)}
    if err is not None:
        d["normwise_err"] = err
    d.update(kw)
    return d


# ------------------------------------------------------------------ configs

def dgemm_1024(R):
    """Plain DGEMM 1024^3, U[-1, 1), error vs the DD oracle over the full C."""
    import oracle
    fg, L = R.fg, R.L
    n = 1024
    rng = np.random.default_rng(SEED)
    a = rng.uniform(-1.0, 1.0, (n, n))
    b = rng.uniform(-1.0, 1.0, (n, n))
    da, db = fg.DeviceArray.from_numpy(a, R.ctx), fg.DeviceArray.from_numpy(b, R.ctx)
    dc = fg.DeviceArray((n, n), np.float64, R.ctx)
    ref = oracle.dd_full(a, b)
    na, nb = oracle.fro(a), oracle.fro(b)
    out = {}
    for name, mode, sl in (("plain", L.FG_MODE_PLAIN, 0), ("split_crt16", L.FG_MODE_SPLIT, 0),
                           ("split_ozaki9", L.FG_MODE_SPLIT, 9)):
        ms = R.time(R.gemm(L.FG_F64, mode, sl, n, n, n, da.ptr, db.ptr, dc.ptr))
        err = oracle.normwise_error(dc.to_numpy(), ref, n, n, na, nb)
        out[name] = _entry(2.0 * n ** 3, ms, err)
    out["err_ferray_cpu"] = oracle.normwise_error(oracle.gemm_f64(a, b), ref, n, n, na, nb)
    out["cpu"] = cpu_rate("f64", n, n, n)
    out["error_over"] = "full C (1024 x 1024) vs double-double"
    return out


def sgemm_sweep(R, sizes=(256, 1024, 2048, 4096)):
    """SGEMM f32 N(0, 1): plain FFMA, 3 x BF16 and 6 x BF16 split per N."""
    import oracle
    fg, L = R.fg, R.L
    out = {}
    for n in sizes:
        rng = np.random.default_rng(SEED + n)
        a = rng.standard_normal((n, n), dtype=np.float32)
        b = rng.standard_normal((n, n), dtype=np.float32)
        da, db = fg.DeviceArray.from_numpy(a, R.ctx), fg.DeviceArray.from_numpy(b, R.ctx)
        dc = fg.DeviceArray((n, n), np.float32, R.ctx)
        rows, cols = oracle.sample_indices(n, n, 128, 128, seed=n)
        ar, bc = a[rows], np.ascontiguousarray(b[:, cols])
        na, nb = oracle.fro(a), oracle.fro(b)
        d = {}
        for name, mode, sl in (("plain", L.FG_MODE_PLAIN, 0), ("split3", L.FG_MODE_SPLIT, 2),
                               ("split6", L.FG_MODE_SPLIT, 3), ("split_f16", L.FG_MODE_SPLIT_F16, 0)):
            ms = R.time(R.gemm(L.FG_F32, mode, sl, n, n, n, da.ptr, db.ptr, dc.ptr))
            err = _err(oracle, dc.to_numpy()[np.ix_(rows, cols)], ar, bc, n, n, na, nb)
            d[name] = _entry(2.0 * n ** 3, ms, err)
        for name in ("split3", "split6", "split_f16"):
            d[name]["speed_over_plain"] = round(d["plain"]["ms"] / d[name]["ms"], 2)
            d[name]["err_over_plain"] = round(d[name]["normwise_err"] / d["plain"]["normwise_err"], 3)
        d["cpu"] = cpu_rate("f32", n, n, n)
        out[str(n)] = d
        del da, db, dc
    return out


def cgemm_4096(R, n=4096):
    """CGEMM c32 at N = 4096, Re and Im N(0, 1): plain (8mnk flops) vs the 3-
    and 6-product BF16 split."""
    import oracle
    torch, fg, L = R.torch, R.fg, R.L
    rng = np.random.default_rng(SEED + 7)
    a = (rng.standard_normal((n, n), dtype=np.float32) + 1j * rng.standard_normal((n, n), dtype=np.float32)
         ).astype(np.complex64)
    b = (rng.standard_normal((n, n), dtype=np.float32) + 1j * rng.standard_normal((n, n), dtype=np.float32)
         ).astype(np.complex64)
    da, db = fg.DeviceArray.from_numpy(a, R.ctx), fg.DeviceArray.from_numpy(b, R.ctx)
    dc = fg.DeviceArray((n, n), np.complex64, R.ctx)
    rows, cols = oracle.sample_indices(n, n, 96, 96, seed=3)
    ar, bc = a[rows], np.ascontiguousarray(b[:, cols])
    na, nb = oracle.fro(a), oracle.fro(b)
    d = {}
    for name, mode, sl in (("plain", L.FG_MODE_PLAIN, 0), ("split3", L.FG_MODE_SPLIT, 2),
                           ("split6", L.FG_MODE_SPLIT, 3), ("split_f16", L.FG_MODE_SPLIT_F16, 0)):
        ms = R.time(R.gemm(L.FG_C32, mode, sl, n, n, n, da.ptr, db.ptr, dc.ptr))
        err = _err(oracle, dc.to_numpy()[np.ix_(rows, cols)], ar, bc, n, n, na, nb)
        d[name] = _entry(8.0 * n ** 3, ms, err)
    for name in ("split3", "split6", "split_f16"):
        d[name]["speed_over_plain"] = round(d["plain"]["ms"] / d[name]["ms"], 2)
        d[name]["err_over_plain"] = round(d[name]["normwise_err"] / d["plain"]["normwise_err"], 3)
    d["cpu"] = cpu_rate("c64", n, n, n)
    del da, db, dc
    torch.cuda.empty_cache()
    return d


def _spread_operand(torch, nn, spread, cplx, gen):
    """diag(10^(s u)) G diag(10^(s v)) on the device, f64 (complex: complex128)."""
    g = torch.randn(nn, nn, dtype=torch.float64, device="cuda", generator=gen)
    if cplx:
        g = torch.complex(g, torch.randn(nn, nn, dtype=torch.float64, device="cuda", generator=gen))
    du = 10.0 ** (spread * (2 * torch.rand(nn, dtype=torch.float64, device="cuda", generator=gen) - 1))
    dv = 10.0 ** (spread * (2 * torch.rand(nn, dtype=torch.float64, device="cuda", generator=gen) - 1))
    return (du[:, None] * g) * dv[None, :]


def _oz_name(s):
    return ("ozaki%d" if s <= 10 else "crt%d") % s


def ozaki_sweep(R, sizes=(2048, 4096, 8192), spreads=(0, 4, 8), slices=(8, 9, 16, 17), cpu=True):
    """DGEMM / ZGEMM: plain FP64 (DMMA) vs INT8-Ozaki per exponent spread:
    scheme I with 8 / 9 slices ("ozaki8", "ozaki9") and scheme II with 16 /
    17 moduli ("crt16", "crt17"); errors vs the DD oracle on a sampled
    64 x 64 block."""
    import oracle
    torch, L = R.torch, R.L
    out = {}
    for nn in sizes:
        for cplx in (False, True):
            for spread in spreads:
                gen = torch.Generator(device="cuda")
                gen.manual_seed(SEED + spread + nn + (1 if cplx else 0))
                a = _spread_operand(torch, nn, spread, cplx, gen)
                b = _spread_operand(torch, nn, spread, cplx, gen)
                c = torch.empty_like(a)
                rows, cols = oracle.sample_indices(nn, nn, 64, 64, seed=13)
                ri, ci = torch.as_tensor(rows, device="cuda"), torch.as_tensor(cols, device="cuda")
                ar = a.index_select(0, ri).cpu().numpy()
                bc = b.index_select(1, ci).contiguous().cpu().numpy()
                ref = oracle.dd_sampled(ar, bc, np.arange(len(rows)), np.arange(len(cols)))
                na = float(torch.linalg.norm(torch.view_as_real(a) if cplx else a))
                nb = float(torch.linalg.norm(torch.view_as_real(b) if cplx else b))
                dt = L.FG_C64 if cplx else L.FG_F64
                flops = (8.0 if cplx else 2.0) * nn ** 3
                entry = {}
                for name, mode, sl in [("plain", L.FG_MODE_PLAIN, 0)] + \
                        [(_oz_name(s), L.FG_MODE_SPLIT, s) for s in slices]:
                    ms = R.time(R.gemm(dt, mode, sl, nn, nn, nn, a.data_ptr(), b.data_ptr(), c.data_ptr()),
                                min_ms=20.0)
                    got = c.index_select(0, ri).index_select(1, ci).cpu().numpy()
                    entry[name] = _entry(flops, ms, oracle.normwise_error(got, ref, nn, nn, na, nb))
                for s in slices:
                    e = entry[_oz_name(s)]
                    e["speed_over_plain"] = round(entry["plain"]["ms"] / e["ms"], 2)
                    e["err_over_plain"] = round(e["normwise_err"] / entry["plain"]["normwise_err"], 3)
                out["%s_%d_spread%d" % ("zgemm" if cplx else "dgemm", nn, spread)] = entry
                del a, b, c
                torch.cuda.empty_cache()
    if cpu:
        out["cpu"] = {"%s_%d" % (nm, nn): cpu_rate(kind, nn, nn, nn, budget_s=1.5)
                      for nn in sizes for nm, kind in (("dgemm", "f64"), ("zgemm", "c128"))}
    return out


def i8_square(R, sizes=(1024, 4096, 8192), int8_peak=None):
    """Square i8 x i8 -> i32, bit-exact on a sampled block."""
    torch, fg, L = R.torch, R.fg, R.L
    out = {}
    for n in sizes:
        gen = torch.Generator(device="cuda")
        gen.manual_seed(SEED + n)
        a = torch.randint(-128, 128, (n, n), dtype=torch.int8, device="cuda", generator=gen)
        b = torch.randint(-128, 128, (n, n), dtype=torch.int8, device="cuda", generator=gen)
        c = torch.empty((n, n), dtype=torch.int32, device="cuda")

        def call():
            st = R.lib.fg_gemm_i8_signed(R.ctx.handle, n, n, n, a.data_ptr(), b.data_ptr(), c.data_ptr(), 0,
                                         R.sh)
            if st != 0:
                raise RuntimeError(R.lib.fg_last_error().decode())
        ms = R.time(call, min_ms=40.0)
        rng = np.random.default_rng(n)
        rows = np.sort(rng.choice(n, 32, replace=False))
        cols = np.sort(rng.choice(n, 32, replace=False))
        ah = a[torch.as_tensor(rows, device="cuda")].cpu().numpy().astype(np.int64)
        bh = b[:, torch.as_tensor(cols, device="cuda")].cpu().numpy().astype(np.int64)
        want = ((ah @ bh + 2 ** 31) % 2 ** 32 - 2 ** 31).astype(np.int32)
        got = c.cpu().numpy()[np.ix_(rows, cols)]
        tops = 2.0 * n ** 3 / ms / 1e9
        v, sp = fg.tune_lookup("i8", n, n, n)
        d = {"tops": round(tops, 1), "ms": round(ms, 4), "frac_of_nominal_dense_int8_4500": round(tops / 4500, 3),
             "variant": v, "splits": sp, "bit_exact_sampled": bool(np.array_equal(got, want)),
             "cpu": cpu_rate("i8", n, n, n)}
        if int8_peak:
            d["frac_of_probe_int8"] = round(tops / int8_peak, 3)
        out[str(n)] = d
        del a, b, c
    torch.cuda.empty_cache()
    return out


def ragged_cpu(dims, budget_s=3.0, seed=SEED):
    """ferray's per-problem loop over a ragged batch (matmul_batched calls one
    GEMM per problem, products/mod.rs:579-659), restated: the oracle's f32
    and i8 GEMMs over a seeded subset of the problems that fits the budget;
    rate = their flops / time."""
    import oracle
    threads = pool_threads()
    oracle.set_threads(threads)
    rng = np.random.default_rng(seed)
    order = rng.permutation(len(dims))
    out = {}
    for kind, gen, fn in (("f32", lambda s: rng.standard_normal(s, dtype=np.float32), oracle.gemm_f32),
                          ("i8", lambda s: rng.integers(-128, 128, s, dtype=np.int8), oracle.gemm_i8_signed)):
        flops, t, done = 0.0, 0.0, 0
        for idx in order:
            m, n, k = (int(x) for x in dims[idx])
            a, b = gen((m, k)), gen((k, n))
            t0 = time.perf_counter()
            fn(a, b)
            t += time.perf_counter() - t0
            flops += 2.0 * m * n * k
            done += 1
            if t > budget_s:
                break
        out[kind] = {"value": round(flops / t / 1e12, 4), "unit": "TOPS" if kind == "i8" else "TFLOP/s",
                     "cores": threads, "kind": "port",
                     "sample": "%d of %d problems, one call each, %.2f s" % (done, len(dims), t),
                     "batch_ms_extrapolated": round(t / flops * sum(2.0 * m * n * k for m, n, k in dims) * 1e3, 1)}
    return out
