"""Parity at N = 4096, where the tuned dispatch picks the large-tile kernel
variants (CTA-pair tcgen05 kernels, cp.async FFMA, DMMA) the smaller parity
cases do not reach.  Floats are checked against the double-double oracle on
a seeded 192 x 192 sample of C (normwise estimate), with the same bounds as
the smaller cases; i8 is bit-exact on a sampled block."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 4096
U64, U32 = 2.0 ** -53, 2.0 ** -24


def _sampled_err(fg, oracle, a, b, c):
    rows, cols = oracle.sample_indices(a.shape[0], b.shape[1], 192, 192, seed=4096)
    return oracle.error_vs_dd(a, b, c, rows, cols)


def test_f32_4096_plain_and_split_forms(fg, oracle):
    r = np.random.default_rng(4096)
    a, b = r.standard_normal((N, N), dtype=np.float32), r.standard_normal((N, N), dtype=np.float32)
    errs = {}
    for form, kw in (("plain", {}), ("split3", {"mode": "split", "bf16_slices": 2}),
                     ("split6", {"mode": "split", "bf16_slices": 3}), ("split_f16", {"mode": "split_f16"})):
        c = np.zeros((N, N), np.float32)
        assert fg.gemm_f32(N, N, N, 1.0, a, b, 0.0, c, **kw)
        errs[form] = _sampled_err(fg, oracle, a, b, c)
    assert errs["plain"] <= N * U32, errs
    assert errs["split3"] <= 2.0 ** -15 + N * U32, errs
    # the 6-product form: no worse than twice the plain FFMA kernel's error
    assert errs["split6"] <= 2 * errs["plain"], errs
    assert errs["split_f16"] <= 2 * errs["plain"], errs


@pytest.mark.parametrize("mode", ["plain", "split"])
def test_f64_4096(fg, oracle, mode):
    r = np.random.default_rng(4097)
    a, b = r.uniform(-1, 1, (N, N)), r.uniform(-1, 1, (N, N))
    c = np.zeros((N, N))
    assert fg.gemm_f64(N, N, N, 1.0, a, b, 0.0, c, mode=mode)
    err = _sampled_err(fg, oracle, a, b, c)
    assert err <= N * U64, (mode, err)


def test_i8_4096_sampled_bit_exact(fg):
    r = np.random.default_rng(4098)
    a = r.integers(-128, 128, (N, N), dtype=np.int8)
    b = r.integers(-128, 128, (N, N), dtype=np.int8)
    c = np.zeros((N, N), np.int32)
    assert fg.gemm_i8_signed(N, N, N, a, b, c)
    rows = np.sort(r.choice(N, 64, replace=False))
    cols = np.sort(r.choice(N, 64, replace=False))
    want = (a[rows].astype(np.int64) @ b[:, cols].astype(np.int64))
    want = ((want + 2 ** 31) % 2 ** 32 - 2 ** 31).astype(np.int32)
    np.testing.assert_array_equal(c[np.ix_(rows, cols)], want)
