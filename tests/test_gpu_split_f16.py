"""Split mode FP16 (FG_MODE_SPLIT_F16): three tcgen05 products of two FP16
slices of the operands scaled by powers of two from their largest
magnitudes.  Checked against the double-double oracle: its error is bounded
by the two-slice representation (about 2^-22 |a||b| per product) plus FP32
accumulation: the tests require at most half the 3 x BF16 form's error, and
against the plain FFMA kernel's at most 4x below K = 1024 and 2.5x from
there (2x at K = 4096 in the large parity test; 0.5x at 8192).  Scaling cases: operands
far outside FP16's range (1e30, 1e-30), mixed magnitudes, zeros, Inf / NaN
propagation, alpha / beta, complex, batches and the split-K path."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

U32 = 2.0 ** -24


def _err(oracle, a, b, c):
    return oracle.error_vs_dd(a, b, c)


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (17, 13, 9), (128, 256, 128), (300, 257, 129),
                                   (1024, 1024, 1024), (2048, 2048, 2048), (64, 96, 8192)])
def test_f16_split_accuracy_vs_plain_and_bf16(fg, oracle, m, n, k):
    r = np.random.default_rng(m + 3 * n + k)
    a = r.standard_normal((m, k)).astype(np.float32)
    b = r.standard_normal((k, n)).astype(np.float32)
    out = {}
    for name, kw in (("f16", {"mode": "split_f16"}), ("plain", {}), ("bf16", {"mode": "split"})):
        c = np.zeros((m, n), np.float32)
        assert fg.gemm_f32(m, n, k, 1.0, a, b, 0.0, c, **kw)
        out[name] = _err(oracle, a, b, c)
    # representation: two FP16 slices leave about 2^-22 |a||b| per product
    assert out["f16"] <= 2.0 ** -21 + k * U32, out
    if k >= 64:
        assert out["f16"] <= out["bf16"] / 2, out
        # the tensor core's accumulation (products summed with truncation
        # inside each MMA) costs more than FFMA's round-to-nearest at short
        # K, while FFMA's own error grows faster with K: the ratio falls
        # from about 2x at K = 1024 to 0.5x at 8192 (K = 4096: the large
        # parity test holds it to 2x)
        assert out["f16"] <= (2.5 if k >= 1024 else 4) * out["plain"], out


@pytest.mark.parametrize("scale_a,scale_b", [(1e30, 1e-30), (1e-30, 1e-5), (3e4, 7e4), (1e-20, 1e20)])
def test_f16_split_scaling_far_outside_fp16_range(fg, oracle, scale_a, scale_b):
    r = np.random.default_rng(11)
    m, n, k = 200, 150, 300
    a = (r.standard_normal((m, k)) * scale_a).astype(np.float32)
    b = (r.standard_normal((k, n)) * scale_b).astype(np.float32)
    c, cp = np.zeros((m, n), np.float32), np.zeros((m, n), np.float32)
    assert fg.gemm_f32(m, n, k, 1.0, a, b, 0.0, c, mode="split_f16")
    assert fg.gemm_f32(m, n, k, 1.0, a, b, 0.0, cp)
    assert np.all(np.isfinite(c))
    # scaling keeps the error what it is for unscaled data: the
    # representation bound, and the same order as plain FFMA's
    e, ep = _err(oracle, a, b, c), _err(oracle, a, b, cp)
    assert e <= 2.0 ** -21 + k * U32, (e, ep)
    assert e <= 8 * ep, (e, ep)


def test_f16_split_mixed_magnitudes_zeros_and_nonfinite(fg, oracle):
    r = np.random.default_rng(12)
    m, n, k = 96, 80, 200
    a = (r.standard_normal((m, k)) * 10.0 ** r.uniform(-6, 6, (m, 1))).astype(np.float32)
    b = r.standard_normal((k, n)).astype(np.float32)
    c = np.zeros((m, n), np.float32)
    assert fg.gemm_f32(m, n, k, 1.0, a, b, 0.0, c, mode="split_f16")
    assert _err(oracle, a, b, c) <= k * U32
    # all-zero operand: exact zeros
    z = np.zeros((m, k), np.float32)
    c[:] = 1.0
    assert fg.gemm_f32(m, n, k, 1.0, z, b, 0.0, c, mode="split_f16")
    assert np.all(c == 0.0)
    # Inf / NaN in A: its row of C is non-finite (Inf, or NaN where a product
    # meets a zero slice); the scaling of the finite entries is unaffected,
    # so every other row keeps its accuracy
    for bad in (np.inf, np.nan):
        a2 = r.standard_normal((m, k)).astype(np.float32)
        a2[:, :3] *= 1e6  # large finite entries would overflow FP16 unscaled
        a2[5, 7] = bad
        assert fg.gemm_f32(m, n, k, 1.0, a2, b, 0.0, c, mode="split_f16")
        assert not np.any(np.isfinite(c[5]))
        keep = np.delete(np.arange(m), 5)
        ok = a2[keep]
        assert np.all(np.isfinite(c[keep]))
        assert _err(oracle, ok, b, np.ascontiguousarray(c[keep])) <= k * U32


def test_f16_split_alpha_beta(fg):
    r = np.random.default_rng(13)
    m, n, k = 130, 300, 77
    a = r.standard_normal((m, k)).astype(np.float32)
    b = r.standard_normal((k, n)).astype(np.float32)
    c0 = r.standard_normal((m, n)).astype(np.float32)
    c = c0.copy()
    assert fg.gemm_f32(m, n, k, 2.0, a, b, 0.5, c, mode="split_f16")
    want = 2.0 * (a.astype(np.float64) @ b.astype(np.float64)) + 0.5 * c0
    assert np.max(np.abs(c - want)) <= 1e-4 * np.max(np.abs(want))


def test_f16_split_complex(fg, oracle):
    r = np.random.default_rng(14)
    m, n, k = 120, 90, 200
    a = (r.standard_normal((m, k)) + 1j * r.standard_normal((m, k))).astype(np.complex64)
    b = (r.standard_normal((k, n)) + 1j * r.standard_normal((k, n))).astype(np.complex64)
    c, cp = np.zeros((m, n), np.complex64), np.zeros((m, n), np.complex64)
    assert fg.gemm_c32(m, n, k, 1.0, 0.0, a, b, 0.0, 0.0, c, mode="split_f16")
    assert fg.gemm_c32(m, n, k, 1.0, 0.0, a, b, 0.0, 0.0, cp)
    e, ep = _err(oracle, a, b, c), _err(oracle, a, b, cp)
    assert e <= 2.0 ** -21 + 2 * k * U32, (e, ep)
    assert e <= 8 * ep, (e, ep)


def test_f16_split_forced_splitk_and_tiles(fg, oracle):
    # every tuned split-f32 tile variant and split-K count reads the same
    # scaling: results within the same bound
    r = np.random.default_rng(15)
    m, n, k = 256, 256, 2048
    a = r.standard_normal((m, k)).astype(np.float32)
    b = r.standard_normal((k, n)).astype(np.float32)
    c0 = np.zeros((m, n), np.float32)
    assert fg.gemm_f32(m, n, k, 1.0, a, b, 0.0, c0, mode="split_f16")
    e0 = _err(oracle, a, b, c0)
    assert e0 <= 2.0 ** -21 + k * U32
    for variant in (0, 1, 2):
        for splits in (1, 4):
            with fg.tune_forced("split_f32", variant, splits):
                c = np.zeros((m, n), np.float32)
                assert fg.gemm_f32(m, n, k, 1.0, a, b, 0.0, c, mode="split_f16")
            # the same products in another tile / K order: the same error level
            assert _err(oracle, a, b, c) <= 2 * e0, (variant, splits)
