"""CPU tests of the C-ABI library: it loads without a GPU and exports every
function include/ferray_gpu.h declares; calls that need no device report
errors the way the header says (no compute is issued)."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ferray_gpu.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fg_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_reference_surface():
    names = declared_functions()
    for want in ("fg_gemm_f64", "fg_gemm_f32", "fg_gemm_c64", "fg_gemm_c32", "fg_gemm_i8",
                 "fg_gemm_i8_signed", "fg_gemm_i16", "fg_quantized_matmul", "fg_matmul",
                 "fg_gemm_batched_strided", "fg_gemm_grouped", "fg_server_start"):
        assert want in names


def test_library_exports_every_declared_symbol():
    from ferray_b200 import _lib
    lib = C.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding declares the same set
    assert set(declared_functions()) <= set(_lib.SIGNATURES)


def test_status_strings_and_errors_without_device():
    from ferray_b200 import _lib
    lib = _lib.load()
    assert lib.fg_status_string(_lib.FG_OK) == b"ok"
    assert lib.fg_status_string(_lib.FG_ERR_SHAPE) == b"shape mismatch"
    # null context / null out pointer are argument errors, not crashes
    assert lib.fg_gemm_f64(None, 0, 0, 1, 1, 1, 1.0, None, None, 0.0, None, None) == _lib.FG_ERR_INVALID
    assert lib.fg_init(0, None) == _lib.FG_ERR_INVALID


def test_init_fails_loudly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from ferray_b200 import _lib
    lib = _lib.load()
    h = C.c_void_p()
    assert lib.fg_init(0, C.byref(h)) != _lib.FG_OK
    assert h.value is None


def test_package_has_no_cpu_fallback(tmp_path, monkeypatch):
    import importlib
    from ferray_b200 import _lib
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "missing.so"))
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(OSError):
        _lib.load()
    importlib.reload(_lib)


def test_tune_table_lookup_and_force_without_device():
    """The autotune table is host data: bucketing, the compiled-in choices
    and forced overrides work without a GPU."""
    import ferray_b200 as fg
    from ferray_b200 import _lib, autotune
    lib = _lib.load()
    n = C.c_int()
    for op, want in zip(range(4), (4, 3, 6, 6)):
        assert lib.fg_tune_variants(op, C.byref(n)) == 0 and n.value == want
    assert lib.fg_tune_variants(9, C.byref(n)) == _lib.FG_ERR_INVALID
    # every shape maps to a valid choice
    for op in fg.TUNE_OPS:
        for m, nn, k in [(1, 1, 1), (128, 129, 8192), (5000, 70, 100000)]:
            v, s = fg.tune_lookup(op, m, nn, k)
            n = C.c_int()
            assert lib.fg_tune_variants(fg.TUNE_OPS[op], C.byref(n)) == 0
            assert 0 <= v < n.value and 1 <= s <= 16
    # forced choices win everywhere, then the table comes back
    before = fg.tune_lookup("i8", 300, 300, 5000)
    with fg.tune_forced("i8", 1, 8):
        assert fg.tune_lookup("i8", 300, 300, 5000) == (1, 8)
        assert fg.tune_lookup("i8", 9000, 9000, 9000) == (1, 8)
    assert fg.tune_lookup("i8", 300, 300, 5000) == before
    assert lib.fg_tune_force(0, 4, 1) == _lib.FG_ERR_INVALID
    assert lib.fg_tune_force(1, 3, 1) == _lib.FG_ERR_INVALID
    assert lib.fg_tune_force(2, 6, 1) == _lib.FG_ERR_INVALID
    assert lib.fg_tune_force(3, 6, 1) == _lib.FG_ERR_INVALID
    assert lib.fg_tune_force(0, 0, 17) == _lib.FG_ERR_INVALID
    # the compiled-in table is the committed include: check one entry per op
    inc = open(os.path.join(ROOT, "ferray_b200", "csrc", "tune_table.inc")).read()
    body = inc[inc.index("= {"):]
    entries = [tuple(map(int, e)) for e in re.findall(r"\{(\d+),(\d+)\}", body)]
    assert len(entries) == 4 * autotune.BUCKETS ** 3
    for oi, op in enumerate(autotune.OPS):
        for (bm, bn, bk) in [(0, 0, 0), (3, 5, 6), (6, 6, 6)]:
            idx = ((oi * autotune.BUCKETS + bm) * autotune.BUCKETS + bn) * autotune.BUCKETS + bk
            m, nn, k = (autotune.REPR[b] for b in (bm, bn, bk))
            assert fg.tune_lookup(op, m, nn, k) == entries[idx]


def test_multi_dot_order_matches_the_reference_programme():
    """The parenthesisation is host logic: fg_multi_dot_order against the
    restated dynamic programme of products/mod.rs:839-855."""
    import numpy as np
    import oracle
    import ferray_b200 as fg
    rng = np.random.default_rng(3)
    for trial in range(40):
        n = int(rng.integers(2, 9))
        dims = [int(x) for x in rng.integers(1, 600, n + 1)]
        want = oracle.chain_order(dims)
        got = fg.multi_dot_order(dims)
        np.testing.assert_array_equal(np.triu(got, 1), np.triu(want, 1))
    # ties keep the first split (all-equal dims)
    assert fg.multi_dot_order([4, 4, 4, 4])[0][2] == oracle.chain_order([4, 4, 4, 4])[0][2]


def _npy_bytes(arr, version=None):
    import io
    import numpy as np
    f = io.BytesIO()
    if version is None:
        np.save(f, arr)
    else:
        np.lib.format.write_array(f, arr, version=version)
    return f.getvalue()


def test_npy_parse_reference_fixture_cases():
    """The dtype cases of fixtures/io/npy_dtypes.json (NumPy 2.4.5 save /
    load), written here by NumPy's own writer: GEMM operand types parse with
    their shape and payload offset, the others are rejected as dtypes, and a
    Fortran-order array reports its order."""
    import json
    import numpy as np
    import ferray_b200 as fg
    cases = json.load(open(os.path.join(ROOT, "tests", "golden", "npy_dtypes.json")))
    gemm_types = {"<f4", "<f8", "|u1", "<c8", "<c16"}
    seen = 0
    for cs in cases:
        data = cs["data"]
        if "complex" in cs["dtype"]:
            data = [complex(re, im) for re, im in data]
        arr = np.array(data, dtype=cs["dtype"]).reshape(cs["shape"])
        if cs.get("fortran_order"):
            arr = np.asfortranarray(arr)
        blob = _npy_bytes(arr)
        if cs["descr"] in gemm_types:
            dt, shape, fortran, off = fg.npy_parse(blob)
            assert dt == arr.dtype and shape == tuple(cs["shape"]), cs["name"]
            assert fortran == bool(cs.get("fortran_order")), cs["name"]
            payload = np.frombuffer(blob[off:], dtype=dt)
            order = "F" if fortran else "C"
            np.testing.assert_array_equal(payload.reshape(shape, order=order), arr)
            seen += 1
        else:
            with pytest.raises(fg.InvalidDtype):
                fg.npy_parse(blob)
    assert seen >= 5


def test_npy_parse_versions_and_malformed_images():
    import numpy as np
    import ferray_b200 as fg
    a = np.arange(12, dtype=np.int16).reshape(3, 4)
    for v in ((1, 0), (2, 0), (3, 0)):
        dt, shape, fo, off = fg.npy_parse(_npy_bytes(a, v))
        assert dt == np.int16 and shape == (3, 4) and not fo
    blob = _npy_bytes(np.zeros((2, 3), np.float32))
    with pytest.raises(fg.InvalidValue):
        fg.npy_parse(b"NOTNPY" + blob[6:])
    with pytest.raises(fg.ShapeMismatch):
        fg.npy_parse(blob[:-4])                         # payload shorter than the shape
    with pytest.raises(fg.InvalidDtype):
        fg.npy_parse(_npy_bytes(np.zeros(3, ">f8")))    # big-endian
    dt, shape, fo, off = fg.npy_parse(_npy_bytes(np.float64(2.5)))  # 0-d
    assert shape == () and dt == np.float64
