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
