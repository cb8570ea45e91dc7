""".npy images straight into device buffers, then a GEMM on them."""
import io

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _npy(arr):
    f = io.BytesIO()
    np.save(f, arr)
    return f.getvalue()


def test_npy_load_then_matmul_f64(fg, oracle):
    r = np.random.default_rng(0)
    a = r.standard_normal((120, 70))
    b = r.standard_normal((70, 50))
    da, db = fg.npy_load(_npy(a)), fg.npy_load(_npy(b))
    assert da.shape == (120, 70) and da.dtype == np.float64
    np.testing.assert_array_equal(da.to_numpy(), a)
    c = fg.matmul(da, db).to_numpy()
    assert oracle.error_vs_dd(a, b, c) <= 70 * 2.0 ** -53


def test_npy_load_i8_exact(fg, oracle):
    r = np.random.default_rng(1)
    a = r.integers(-128, 128, (33, 300), dtype=np.int8)
    b = r.integers(-128, 128, (300, 17), dtype=np.int8)
    da, db = fg.npy_load(_npy(a)), fg.npy_load(_npy(b))
    c = fg.DeviceArray((33, 17), np.int32)
    assert fg.gemm_i8_signed(33, 17, 300, da, db, c)
    np.testing.assert_array_equal(c.to_numpy(), oracle.gemm_i8_signed(a, b))


def test_npy_load_rejects_fortran_order(fg):
    with pytest.raises(fg.Unsupported):
        fg.npy_load(_npy(np.asfortranarray(np.zeros((3, 4)))))


def _npz(compressed, **arrays):
    f = io.BytesIO()
    (np.savez_compressed if compressed else np.savez)(f, **arrays)
    return f.getvalue()


@pytest.mark.parametrize("compressed", [False, True])
def test_npz_load_every_operand_type(fg, compressed):
    r = np.random.default_rng(2)
    arrays = {"f64": r.standard_normal((5, 7)), "f32": r.standard_normal((3, 9)).astype(np.float32),
              "c128": (r.standard_normal((4, 4)) + 1j * r.standard_normal((4, 4))),
              "c64": (r.standard_normal((2, 3)) + 1j).astype(np.complex64),
              "i8": r.integers(-128, 128, (6, 6), dtype=np.int8), "u8": r.integers(0, 256, (6,), dtype=np.uint8),
              "i16": r.integers(-2 ** 15, 2 ** 15, (3, 5), dtype=np.int16),
              "f16": r.standard_normal((8, 2)).astype(np.float16)}
    data = _npz(compressed, **arrays)
    assert fg.npz_names(data) == list(arrays)
    for name, want in arrays.items():
        got = fg.npz_load(data, name)
        assert got.shape == want.shape
        np.testing.assert_array_equal(got.to_numpy().view(want.dtype), want)


def test_npz_load_then_split_sgemm(fg, oracle):
    r = np.random.default_rng(3)
    a = r.standard_normal((200, 96)).astype(np.float32)
    b = r.standard_normal((96, 150)).astype(np.float32)
    data = _npz(True, a=a, b=b)
    c = fg.matmul(fg.npz_load(data, "a"), fg.npz_load(data, "b"), mode="split").to_numpy()
    assert oracle.error_vs_dd(a, b, c) <= 1e-6


def test_npz_load_errors(fg):
    data = _npz(False, x=np.arange(3, dtype=np.int32), y=np.zeros(2))
    with pytest.raises(fg.InvalidDtype):  # i32 is no GEMM operand type (the npy rule)
        fg.npz_load(data, "x")
    with pytest.raises(fg.FerrayError):
        fg.npz_load(data, "missing")
