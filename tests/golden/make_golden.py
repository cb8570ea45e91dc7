"""Generate the golden fixtures under tests/golden/ from the ferray sources.

Run with the environment variable FERRAY_ROOT set to a checkout of the
ferray workspace; the JSON files it writes are committed, so nothing at test
time reads the ferray tree.

Fixtures:

* ``matmul_numpy.json`` -- the NumPy 2.4.5 known answers of
  fixtures/linalg/matmul.json (ferray-linalg/tests/oracle.rs:118-138 loads the
  same file), copied case by case.
* ``gemm_hexfloat.json`` -- the exact NumPy ``@`` results written as hex floats
  in ferray-linalg/src/gemm/mod.rs:1213-1275 (cancellation row, 4x3x5 random
  case), parsed from the source text.
* ``integer_cases.json`` -- the deterministic operand formulas of
  ferray-linalg/src/gemm/integer_tests.rs:65-414 (i16, i8 x i8, quantized,
  including i8::MIN/MAX at odd sizes and accumulate mode), evaluated with Rust
  `as i8`/`as i16`/`as u8` wrapping, with the answers of the naive
  wrapping-i32 loops those tests assert equality against
  (integer_tests.rs:15-63).
* ``npy_dtypes.json`` -- the save / load cases of fixtures/io/npy_dtypes.json
  (NumPy 2.4.5): data, shape, dtype, descr and Fortran order per case (complex
  values as [re, im] pairs); the tests write them with NumPy's own .npy
  writer and parse the bytes.
"""
import json
import os
import re

import numpy as np

FERRAY_ROOT = os.environ.get("FERRAY_ROOT", "")
HERE = os.path.dirname(os.path.abspath(__file__))


def wrap(v, bits, signed=True):
    v = int(v) & ((1 << bits) - 1)
    if signed and v >= 1 << (bits - 1):
        v -= 1 << bits
    return v


def hexf(s):
    return float.fromhex(s)


def matmul_numpy():
    src = json.load(open(os.path.join(FERRAY_ROOT, "fixtures/linalg/matmul.json")))
    cases = []
    for tc in src["test_cases"]:
        cases.append({
            "name": tc["name"],
            "a": tc["inputs"]["a"]["data"], "a_shape": tc["inputs"]["a"]["shape"],
            "b": tc["inputs"]["b"]["data"], "b_shape": tc["inputs"]["b"]["shape"],
            "expected": tc["expected"]["data"], "expected_shape": tc["expected"]["shape"],
            "tolerance_ulps": tc.get("tolerance_ulps", 0),
        })
    return {"numpy_version": src.get("numpy_version"), "source": "fixtures/linalg/matmul.json",
            "cases": cases}


def gemm_hexfloat():
    text = open(os.path.join(FERRAY_ROOT, "ferray-linalg/src/gemm/mod.rs")).read()
    out = []
    for name, shape_a, shape_b in (("gemm_matches_numpy_cancellation", (2, 3), (3, 2)),
                                   ("gemm_matches_numpy_random_4x3x5", (4, 3), (3, 5))):
        body = text[text.index("fn " + name):]
        body = body[:body.index("#[test]")] if "#[test]" in body else body
        # a / b / expected blocks are `vec![...]` / `[...]` literals in order.
        blocks = re.findall(r"(?:vec!\[|expected = \[)(.*?)\]", body, re.S)
        vals = []
        for blk in blocks[:3]:
            items = re.findall(r'hexf64\("([^"]+)"\)|(-?\d+\.\d+)', blk)
            vals.append([hexf(h) if h else float(d) for h, d in items])
        a, b, exp = vals
        assert len(a) == shape_a[0] * shape_a[1] and len(b) == shape_b[0] * shape_b[1]
        out.append({"name": name, "a": [x.hex() for x in a], "a_shape": list(shape_a),
                    "b": [x.hex() for x in b], "b_shape": list(shape_b),
                    "expected": [x.hex() for x in exp],
                    "max_ulps": 0 if "cancellation" in name else 2,
                    "source": "ferray-linalg/src/gemm/mod.rs"})
    return out


def naive_wrap(a, b, m, n, k):
    A = np.array(a, np.int64).reshape(m, k)
    B = np.array(b, np.int64).reshape(k, n)
    C = A @ B
    return [wrap(v, 32) for v in C.reshape(-1)]


def integer_cases():
    cases = []

    def add(kind, name, m, n, k, a, b, c0=None, **extra):
        if kind in ("i16", "i8s"):
            exp = naive_wrap(a, b, m, n, k)
            if c0 is not None:
                exp = [wrap(x + y, 32) for x, y in zip(exp, c0)]
        else:
            exp = None
        d = {"kind": kind, "name": name, "m": m, "n": n, "k": k, "a": a, "b": b,
             "c0": c0, "expected": exp}
        d.update(extra)
        cases.append(d)

    # integer_tests.rs:66-86
    m, n, k = 12, 24, 16
    add("i16", "gemm_i16_matches_naive_at_kernel_sizes", m, n, k,
        [wrap(i * 17 - 200, 16) for i in range(m * k)], [wrap(i * 13 - 100, 16) for i in range(k * n)])
    # :88-109
    m, n, k = 7, 11, 9
    add("i16", "gemm_i16_handles_odd_dims_and_k", m, n, k,
        [wrap(i * 23 + 5, 16) for i in range(m * k)], [wrap(i * 19 - 60, 16) for i in range(k * n)])
    # :111-136
    m, n, k = 8, 8, 8
    add("i16", "gemm_i16_accumulate_preserves_existing_c", m, n, k,
        [wrap(i * 2, 16) for i in range(m * k)], [wrap(i * 3, 16) for i in range(k * n)],
        c0=[i * 1000 for i in range(m * n)])
    # :138-159
    m, n, k = 12, 16, 20
    add("i8s", "gemm_i8_signed_matches_naive", m, n, k,
        [wrap(i * 7 - 60, 8) for i in range(m * k)], [wrap(i * 11 - 80, 8) for i in range(k * n)])
    # :161-200
    m, n, k = 13, 17, 19

    def ea(i):
        r = i % 6
        return [-128, 127, -127, 1, -1, wrap(i * 5 - 80, 8)][r]

    def eb(i):
        r = i % 5
        return [127, -128, 0, wrap(i * 3 - 50, 8), wrap(i * 3 - 50, 8)][r]
    add("i8s", "gemm_i8_signed_extreme_values_through_entry", m, n, k,
        [ea(i) for i in range(m * k)], [eb(i) for i in range(k * n)])
    # :202-225
    m, n, k = 8, 8, 12
    add("i8s", "gemm_i8_signed_accumulate_through_entry", m, n, k,
        [wrap(i * 3 - 30, 8) for i in range(m * k)], [wrap(i * 5 - 40, 8) for i in range(k * n)],
        c0=[i * 100 for i in range(m * n)])
    # :227-264
    m, n, k = 9, 13, 11
    add("i8s", "gemm_i8_signed_negative_inputs", m, n, k,
        [-(i % 100) if i % 2 == 0 else (i % 100) for i in range(m * k)],
        [-(i % 80) if i % 3 == 0 else (i % 80) for i in range(k * n)])
    # quantized: :266-311, :313-364, :366-414 (float answers computed by the
    # oracle restatement at test time; the reference asserts rel < 1e-5/1e-4).
    m, n, k = 8, 12, 16
    add("qmm", "quantized_matmul_zero_zero_points_matches_scaled_gemm_i8", m, n, k,
        [wrap(i * 7 + 3, 8, False) & 0x7F for i in range(m * k)],
        [wrap(i * 11 - 50, 8) for i in range(k * n)], a_zp=0, b_zp=0, scale_a=0.01,
        scale_b=0.02, rel_tol=1e-5)
    m, n, k = 10, 14, 18
    add("qmm", "quantized_matmul_with_nonzero_zero_points", m, n, k,
        [wrap(i * 13, 8, False) & 0x7F for i in range(m * k)],
        [wrap(i * 7 - 40, 8) for i in range(k * n)], a_zp=64, b_zp=-3, scale_a=0.0078,
        scale_b=0.015, rel_tol=1e-4)
    m, n, k = 6, 10, 12
    add("qmm", "quantized_matmul_accumulate", m, n, k,
        [wrap(i * 5, 8, False) & 0x3F for i in range(m * k)],
        [wrap(i - 30, 8) for i in range(k * n)], a_zp=64, b_zp=0, scale_a=0.05,
        scale_b=0.05, c0_f32=[i * 0.1 for i in range(m * n)], rel_tol=1e-4)
    return cases


def npy_dtypes():
    d = json.load(open(os.path.join(FERRAY_ROOT, "fixtures", "io", "npy_dtypes.json")))
    assert d["numpy_version"] == "2.4.5"
    out = []
    for c in d["test_cases"]:
        inp = c["inputs"]
        data = inp["data"]["data"]
        if data and isinstance(data[0], dict):
            data = [[v["re"], v["im"]] for v in data]
        out.append({"name": c["name"], "data": data, "shape": inp["data"]["shape"],
                    "dtype": inp["data"]["dtype"], "descr": inp.get("numpy_dtype_str", "<f8"),
                    "fortran_order": bool(inp.get("fortran_order", False))})
    return out


def main():
    with open(os.path.join(HERE, "matmul_numpy.json"), "w") as f:
        json.dump(matmul_numpy(), f, indent=1)
    with open(os.path.join(HERE, "gemm_hexfloat.json"), "w") as f:
        json.dump(gemm_hexfloat(), f, indent=1)
    with open(os.path.join(HERE, "integer_cases.json"), "w") as f:
        json.dump(integer_cases(), f)
    with open(os.path.join(HERE, "npy_dtypes.json"), "w") as f:
        json.dump(npy_dtypes(), f, indent=1)
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    if not FERRAY_ROOT or not os.path.isdir(FERRAY_ROOT):
        raise SystemExit("set FERRAY_ROOT to a checkout of the ferray workspace")
    main()
