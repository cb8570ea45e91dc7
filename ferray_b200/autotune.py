"""Autotuner of the GEMM dispatch table (csrc/tune_table.inc, tune_table.json).

Every tuned family ("op") has kernel variants (tile shape / pipeline depth)
and a split-K count.  For each bucket triple of (M, N, K) -- buckets
<=16, <=32, ..., <=4096, >4096 -- the tuner times every candidate on the
bucket's representative shape (its upper bound; 8192 for the last bucket)
and keeps the fastest one whose result agrees with the untuned kernel
(integers bit-exact, floats to a normwise 1e-5 / 1e-13).

Candidates: every variant; split-K counts 2, 4, 8, 16 where the variant's
output tiles (or thread blocks) are fewer than twice the SM count and K
holds at least that many split units.  Timing: one warm-up call, then the
best of three repetitions of R back-to-back calls on the context stream
bracketed by fg_sync (R chosen so one repetition lasts >= 2 ms), so launch
and split-K combine costs count like they do for a caller.

Usage, on the target GPU:
    python -m ferray_b200.autotune --out DIR [--ops i8,split_f32,f64,f32]
writes DIR/tune_candidates.json (every candidate's time), DIR/tune_table.json
(per bucket: the choice, untuned and tuned time) and DIR/tune_table.inc.  Copy both into ferray_b200/ and ferray_b200/csrc/ and
rebuild to compile the table in.  `python -m ferray_b200.autotune
--default DIR` writes the untuned table (variant 0, no split everywhere).
"""
import argparse
import ctypes as C
import datetime
import json
import os
import time

import numpy as np

OPS = ["i8", "split_f32", "f64", "f32"]
BUCKETS = 10
REPR = [16, 32, 64, 128, 256, 512, 1024, 2048, 4096, 8192]
SPLITS = [1, 2, 4, 8, 16]
MARGIN = 1.03  # a candidate must beat the untuned kernel by 3%
# tile edge per variant (output tiles per block row / column)
TILES = {"i8": [(128, 256), (128, 128), (256, 256), (256, 512)], "split_f32": [(128, 128), (128, 64), (256, 128)],
         "f64": [(128, 128), (64, 64), (32, 128), (128, 32), (128, 128), (32, 256)],
         "f32": [(128, 128), (64, 64), (32, 128), (128, 32), (128, 128), (32, 256)]}
# K per split unit: one tcgen05 K block, or the SIMT split granularity
KUNIT = {"i8": 128, "split_f32": 64, "f64": 64, "f32": 64}


def write_inc(choice, path, meta):
    """choice[op][bm][bn][bk] = (variant, splits) -> C++ table include."""
    lines = ["// tune_table.inc -- generated by ferray_b200/autotune.py; do not edit.",
             "// " + meta,
             "// kTuneTable[op][M bucket][N bucket][K bucket] = {variant, splits};",
             "// ops: " + ", ".join(OPS) + "; buckets <=16, <=32, <=64, <=128, <=256, <=512,"
             " <=1024, <=2048, <=4096, >4096.",
             "constexpr TuneEntry kTuneTable[TUNE_OPS][TUNE_BUCKETS][TUNE_BUCKETS][TUNE_BUCKETS] = {"]
    for op in OPS:
        lines.append("    {  // " + op)
        for bm in range(BUCKETS):
            rows = []
            for bn in range(BUCKETS):
                rows.append("{" + ",".join("{%d,%d}" % tuple(choice[op][bm][bn][bk])
                                           for bk in range(BUCKETS)) + "}")
            lines.append("        {" + ", ".join(rows) + "},")
        lines.append("    },")
    lines.append("};")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def default_choice():
    return {op: [[[(0, 1)] * BUCKETS for _ in range(BUCKETS)] for _ in range(BUCKETS)]
            for op in OPS}


class _Bench:
    """Operands sized for the largest bucket, reused by every shape."""

    def __init__(self, fg, L, op, ctx):
        self.fg, self.L, self.op, self.ctx, self.lib = fg, L, op, ctx, ctx._lib
        rng = np.random.default_rng(42)
        big = REPR[-1] * REPR[-1]
        if op == "i8":
            self.dt, self.odt, self.fgdt = np.int8, np.int32, L.FG_I8
            mk = lambda: rng.integers(-128, 128, big, dtype=np.int8)
        elif op in ("split_f32", "f32"):
            self.dt = self.odt = np.float32
            self.fgdt = L.FG_F32
            mk = lambda: rng.standard_normal(big, dtype=np.float32)
        else:
            self.dt = self.odt = np.float64
            self.fgdt = L.FG_F64
            mk = lambda: rng.standard_normal(big)
        self.mode = L.FG_MODE_SPLIT if op == "split_f32" else L.FG_MODE_PLAIN
        self.a = fg.DeviceArray.from_numpy(mk(), ctx)
        self.b = fg.DeviceArray.from_numpy(mk(), ctx)
        self.c = fg.DeviceArray((big,), self.odt, ctx)
        st = C.c_double if self.dt == np.float64 else C.c_float
        self.one = (st * 2)(1.0, 0.0)
        self.zero = (st * 2)(0.0, 0.0)

    def call(self, m, n, k):
        st = self.lib.fg_gemm(self.ctx.handle, self.fgdt, self.mode, 0, m, n, k, self.one,
                              self.a.ptr, k, self.b.ptr, n, self.zero, self.c.ptr, n, 0, None)
        if st != 0:
            raise RuntimeError(self.lib.fg_last_error().decode())

    def result(self, m, n):
        out = np.empty(m * n, self.odt)
        self.lib.fg_download(self.ctx.handle, out.ctypes.data, self.c.ptr, out.nbytes, None)
        self.ctx.sync()
        return out

    def time(self, m, n, k):
        self.call(m, n, k)
        self.ctx.sync()
        t0 = time.perf_counter()
        self.call(m, n, k)
        self.ctx.sync()
        one = max(time.perf_counter() - t0, 1e-6)
        reps = max(1, min(2000, int(2e-3 / one)))
        best = float("inf")
        for _ in range(3):
            t0 = time.perf_counter()
            for _ in range(reps):
                self.call(m, n, k)
            self.ctx.sync()
            best = min(best, (time.perf_counter() - t0) / reps)
        return best

    def free(self):
        for x in (self.a, self.b, self.c):
            x.free()


def _agree(op, ref, got, k):
    """Integers bit-exact; floats within tol * sqrt(k) * ||ref||_F, which for
    N(0,1) operands is tol * ||A||_F ||B||_F, the normwise scale."""
    if op == "i8":
        return bool(np.array_equal(ref, got))
    tol = 1e-13 if op == "f64" else 1e-5
    den = max(float(np.linalg.norm(ref.astype(np.float64))), 1e-300) * np.sqrt(k)
    return float(np.linalg.norm((got - ref).astype(np.float64))) <= tol * den


def tune_op(fg, L, ctx, op, sm_count, log):
    lib = ctx._lib
    opi = OPS.index(op)
    nvar = C.c_int()
    lib.fg_tune_variants(opi, C.byref(nvar))
    bench = _Bench(fg, L, op, ctx)
    choice = [[[(0, 1)] * BUCKETS for _ in range(BUCKETS)] for _ in range(BUCKETS)]
    records = []
    try:
        for bm in range(BUCKETS):
            for bn in range(BUCKETS):
                for bk in range(BUCKETS):
                    m, n, k = REPR[bm], REPR[bn], REPR[bk]
                    lib.fg_tune_force(opi, 0, 1)
                    bench.call(m, n, k)
                    ref = bench.result(m, n)
                    cands = []
                    for v in range(nvar.value):
                        tm, tn = TILES[op][v]
                        tiles = -(-m // tm) * -(-n // tn)
                        for s in SPLITS:
                            if s > 1 and (tiles >= 2 * sm_count or k // KUNIT[op] < s):
                                continue
                            lib.fg_tune_force(opi, v, s)
                            t = bench.time(m, n, k)
                            ok = (v, s) == (0, 1) or _agree(op, ref, bench.result(m, n), k)
                            cands.append({"variant": v, "splits": s, "ms": round(t * 1e3, 5),
                                          "agrees": bool(ok)})
                    base = next(c for c in cands if (c["variant"], c["splits"]) == (0, 1))
                    best = min((c for c in cands if c["agrees"]), key=lambda c: c["ms"])
                    if best["ms"] * MARGIN >= base["ms"]:
                        best = base  # within timing noise: keep the untuned kernel
                    choice[bm][bn][bk] = (best["variant"], best["splits"])
                    records.append({"m": m, "n": n, "k": k, "candidates": cands,
                                    "choice": [best["variant"], best["splits"]],
                                    "untuned_ms": base["ms"], "tuned_ms": best["ms"],
                                    "rejected": sum(1 for c in cands if not c["agrees"])})
                    log("%s m=%d n=%d k=%d -> variant %d splits %d (%.3fx)" %
                        (op, m, n, k, best["variant"], best["splits"], base["ms"] / best["ms"]))
    finally:
        lib.fg_tune_force(opi, -1, 1)
        bench.free()
    return choice, records


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=".")
    ap.add_argument("--ops", default=",".join(OPS))
    ap.add_argument("--default", action="store_true", help="write the untuned table")
    ap.add_argument("--merge", default=None,
                    help="tune_table.json whose choices are kept for the ops not retuned")
    args = ap.parse_args(argv)
    os.makedirs(args.out, exist_ok=True)
    if args.default:
        write_inc(default_choice(), os.path.join(args.out, "tune_table.inc"),
                  "untuned default: variant 0, no split-K")
        return
    import ferray_b200 as fg
    from ferray_b200 import _lib as L
    ctx = fg.Context(0)
    info = ctx.info()
    import subprocess
    try:
        gpu = subprocess.run(["nvidia-smi", "--query-gpu=name,driver_version", "--format=csv,noheader"],
                             capture_output=True, text=True).stdout.strip().splitlines()[0]
    except Exception:
        gpu = "unknown"
    choice = default_choice()
    report = {"gpu": gpu, "sm_count": info["sm_count"],
              "date": datetime.datetime.utcnow().strftime("%Y-%m-%d %H:%M UTC"),
              "buckets": REPR, "ops": {}}
    if args.merge:
        old = json.load(open(args.merge))
        for op, rows in old["ops"].items():
            if op in args.ops.split(","):
                continue
            recs = []
            for r in rows:
                m, n, k, v, sp = r[:5]
                choice[op][REPR.index(m)][REPR.index(n)][REPR.index(k)] = (v, sp)
                recs.append(r)
            report["ops"][op] = recs
        report["merged_from"] = {"date": old.get("date"), "ops": sorted(report["ops"])}
    t0 = time.time()
    for op in args.ops.split(","):
        choice[op], recs = tune_op(fg, L, ctx, op, info["sm_count"], print)
        report["ops"][op] = recs
    report["seconds"] = round(time.time() - t0, 1)
    with open(os.path.join(args.out, "tune_candidates.json"), "w") as f:
        json.dump(report, f)
    # compact copy (committed beside the table): per bucket the choice and
    # the untuned / tuned times
    compact = dict(report)
    compact["ops"] = {op: [r if isinstance(r, list) else
                           [r["m"], r["n"], r["k"], r["choice"][0], r["choice"][1],
                            r["untuned_ms"], r["tuned_ms"], len(r["candidates"]), r["rejected"]]
                           for r in recs] for op, recs in report["ops"].items()}
    compact["columns"] = ["m", "n", "k", "variant", "splits", "untuned_ms", "tuned_ms",
                          "candidates", "rejected"]
    with open(os.path.join(args.out, "tune_table.json"), "w") as f:
        json.dump(compact, f, separators=(",", ":"))
    write_inc(choice, os.path.join(args.out, "tune_table.inc"),
              "tuned on %s (%d SMs), %s" % (gpu, info["sm_count"], report["date"]))
    ctx.close()


if __name__ == "__main__":
    main()
