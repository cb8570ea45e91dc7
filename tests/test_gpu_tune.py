"""Every autotuned kernel variant and split-K count, forced, against the
oracle: integers bit-exact, floats within the normwise bounds of the plain
and split paths (test_gpu_parity.py states them), including alpha / beta,
accumulate and broadcast batches, so any table the tuner writes is correct
by construction."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

U64, U32 = 2.0 ** -53, 2.0 ** -24
SPLITS = [1, 2, 3, 16]
SHAPES = [(1, 1, 1), (70, 33, 300), (128, 128, 1024), (130, 200, 2100)]
_DD = {}


def dd(oracle, a, b, key):
    """double-double A@B, computed once per input set"""
    if key not in _DD:
        _DD[key] = oracle.dd_full(a, b)
    return _DD[key]


def rng(seed=0):
    return np.random.default_rng(seed)


@pytest.mark.parametrize("variant", [0, 1, 2, 3])
@pytest.mark.parametrize("splits", SPLITS)
@pytest.mark.parametrize("m,n,k", SHAPES + [(300, 520, 700), (257, 129, 4096), (513, 1100, 384)])
def test_i8_variants_bit_exact(fg, oracle, variant, splits, m, n, k):
    r = rng(m + n + k)
    a = r.integers(-128, 128, (m, k), dtype=np.int8)
    b = r.integers(-128, 128, (k, n), dtype=np.int8)
    c0 = r.integers(-2 ** 31, 2 ** 31, (m, n), dtype=np.int64).astype(np.int32)
    with fg.tune_forced("i8", variant, splits):
        c = np.zeros((m, n), np.int32)
        assert fg.gemm_i8_signed(m, n, k, a, b, c)
        np.testing.assert_array_equal(c, oracle.gemm_i8_signed(a, b))
        c = c0.copy()
        assert fg.gemm_i8_signed(m, n, k, a, b, c, accumulate=True)
        np.testing.assert_array_equal(c, oracle.gemm_i8_signed(a, b, c=c0, accumulate=True))
        au = r.integers(0, 256, (m, k), dtype=np.uint8)
        c = np.zeros((m, n), np.int32)
        assert fg.gemm_i8(m, n, k, au, b, c)
        np.testing.assert_array_equal(c, oracle.gemm_i8(au, b, variant="vnni"))


@pytest.mark.parametrize("variant,splits", [(0, 4), (1, 3), (2, 1), (2, 2), (3, 1), (3, 3)])
def test_i8_split_broadcast_batch(fg, oracle, variant, splits):
    r = rng(9)
    a = r.integers(-128, 128, (3, 1, 40, 520), dtype=np.int8)
    b = r.integers(-128, 128, (2, 520, 72), dtype=np.int8)
    want = np.einsum("...ik,...kj->...ij", a.astype(np.int64), b.astype(np.int64))
    want = ((want + 2 ** 31) % 2 ** 32 - 2 ** 31).astype(np.int32)
    with fg.tune_forced("i8", variant, splits):
        got = fg.matmul(fg.DeviceArray.from_numpy(a), fg.DeviceArray.from_numpy(b)).to_numpy()
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("variant", [0, 1, 2])
@pytest.mark.parametrize("splits", SPLITS)
@pytest.mark.parametrize("m,n,k", SHAPES + [(300, 200, 700)])
def test_split_f32_variants(fg, oracle, variant, splits, m, n, k):
    r = rng(m * 3 + k)
    a = r.standard_normal((m, k), dtype=np.float32)
    b = r.standard_normal((k, n), dtype=np.float32)
    c0 = r.standard_normal((m, n), dtype=np.float32)
    with fg.tune_forced("split_f32", variant, splits):
        c = np.zeros((m, n), np.float32)
        assert fg.gemm_f32(m, n, k, 1.0, a, b, 0.0, c, mode="split")
        exact = dd(oracle, a, b, ("s", m, n, k))
        scale = np.linalg.norm(a.astype(np.float64)) * np.linalg.norm(b.astype(np.float64))
        assert np.linalg.norm(c - exact) / scale <= 2.0 ** -15 + k * U32
        c = c0.copy()
        assert fg.gemm_f32(m, n, k, 0.5, a, b, -2.0, c, mode="split")
        ref = 0.5 * exact - 2.0 * c0.astype(np.float64)
        # plus the rounding of the f32 output itself (|C| ~ |beta C0| here)
        assert np.linalg.norm(c - ref) <= ((2.0 ** -15 + (k + 4) * U32) * scale
                                           + 2 * U32 * np.linalg.norm(ref))


@pytest.mark.parametrize("op,dt,u,variant", [("f64", np.float64, U64, v) for v in range(6)] +
                         [("f32", np.float32, U32, v) for v in range(6)])
@pytest.mark.parametrize("splits", SPLITS)
@pytest.mark.parametrize("m,n,k", SHAPES + [(257, 300, 501)])
def test_plain_variants(fg, oracle, op, dt, u, variant, splits, m, n, k):
    r = rng(m + 5 * n)
    a = r.uniform(-1, 1, (m, k)).astype(dt)
    b = r.uniform(-1, 1, (k, n)).astype(dt)
    c0 = r.uniform(-1, 1, (m, n)).astype(dt)
    gemm = fg.gemm_f64 if dt == np.float64 else fg.gemm_f32
    with fg.tune_forced(op, variant, splits):
        c = np.zeros((m, n), dt)
        assert gemm(m, n, k, 1.0, a, b, 0.0, c)
        exact = dd(oracle, a, b, (op, m, n, k))
        scale = np.linalg.norm(a.astype(np.float64)) * np.linalg.norm(b.astype(np.float64))
        assert np.linalg.norm(c - exact) / scale <= k * u
        c = c0.copy()
        assert gemm(m, n, k, 0.5, a, b, 2.0, c)
        ref = 0.5 * exact + 2.0 * c0.astype(np.float64)
        assert np.linalg.norm(c - ref) <= (k + 4) * u * scale + 2 * u * np.linalg.norm(ref)


@pytest.mark.parametrize("variant,splits", [(0, 2), (1, 4), (4, 1), (4, 3)])
def test_plain_split_broadcast_batch(fg, oracle, variant, splits):
    r = rng(4)
    a = r.uniform(-1, 1, (2, 3, 33, 700))
    b = r.uniform(-1, 1, (3, 700, 45))
    with fg.tune_forced("f64", variant, splits):
        got = fg.matmul(fg.DeviceArray.from_numpy(a), fg.DeviceArray.from_numpy(b)).to_numpy()
    want = np.matmul(a, b)
    assert np.max(np.abs(got - want)) <= 700 * U64 * 700


def test_default_table_choices_are_valid_on_device(fg):
    # every bucket's compiled-in choice runs and agrees with the forced baseline
    r = rng(1)
    m, n, k = 100, 90, 2000
    a = r.integers(-128, 128, (m, k), dtype=np.int8)
    b = r.integers(-128, 128, (k, n), dtype=np.int8)
    c1 = np.zeros((m, n), np.int32)
    c2 = np.zeros((m, n), np.int32)
    assert fg.gemm_i8_signed(m, n, k, a, b, c1)
    with fg.tune_forced("i8", 0, 1):
        assert fg.gemm_i8_signed(m, n, k, a, b, c2)
    np.testing.assert_array_equal(c1, c2)


@pytest.mark.parametrize("m,n,k", [(70, 33, 300), (300, 520, 700), (513, 257, 1100)])
@pytest.mark.parametrize("dt", [np.float64, np.complex128])
def test_ozaki_groups_pair_kernel_bitwise_equal(fg, oracle, m, n, k, dt):
    """The Ozaki slice groups are exact int32 GEMMs with the same FP64
    epilogue in the same group order on either kernel, so the single-CTA and
    the CTA-pair group kernels must give bit-identical results."""
    r = rng(m + k)
    a = r.standard_normal((m, k))
    b = r.standard_normal((k, n))
    c0 = r.standard_normal((m, n))
    if dt == np.complex128:
        a = a + 1j * r.standard_normal((m, k))
        b = b + 1j * r.standard_normal((k, n))
        c0 = c0 + 1j * r.standard_normal((m, n))
    outs = []
    for v in (0, 2):
        with fg.tune_forced("i8", v, 1):
            c = c0.copy()
            if dt == np.float64:
                assert fg.gemm_f64(m, n, k, 0.75, a, b, 0.5, c, mode="split")
            else:
                assert fg.gemm_c64(m, n, k, 0.75, 0.0, a, b, 0.5, 0.0, c, mode="split")
            outs.append(c)
    np.testing.assert_array_equal(outs[0], outs[1])
    ref = 0.75 * oracle.dd_full(a, b) + 0.5 * c0
    scale = np.linalg.norm(a) * np.linalg.norm(b)
    assert np.linalg.norm(outs[1] - ref) / scale <= 4 * k * U64


@pytest.mark.parametrize("splits", [1, 3])
@pytest.mark.parametrize("m,n,k", [(130, 48, 77), (257, 45, 300), (64, 260, 1000), (1, 7, 5), (32, 600, 2000)])
def test_ffma_cp_async_kernel_bit_identical(fg, m, n, k, splits):
    """f32 variants 4 and 5 (cp.async ring, A transposed into scratch, B in
    place or packed; 128 x 128 and skinny 32 x 256 tiles) keep the per-output
    k order of variant 0: same bits."""
    r = rng(m * 3 + n + k)
    a = r.standard_normal((m, k)).astype(np.float32)
    b = r.standard_normal((k, n)).astype(np.float32)
    c0 = r.standard_normal((m, n)).astype(np.float32)
    out = []
    for variant in (0, 4, 5):
        with fg.tune_forced("f32", variant, splits):
            c = c0.copy()
            assert fg.gemm_f32(m, n, k, 0.75, a, b, -1.5, c)
            out.append(c)
    np.testing.assert_array_equal(out[0], out[1])
    np.testing.assert_array_equal(out[0], out[2])


@pytest.mark.parametrize("n", [45, 48])
def test_ffma_cp_async_broadcast_batch(fg, n):
    r = rng(n)
    a = r.standard_normal((2, 3, 33, 700)).astype(np.float32)
    b = r.standard_normal((3, 700, n)).astype(np.float32)
    res = []
    for variant in (0, 4):
        with fg.tune_forced("f32", variant, 1):
            res.append(fg.matmul(fg.DeviceArray.from_numpy(a), fg.DeviceArray.from_numpy(b)).to_numpy())
    np.testing.assert_array_equal(res[0], res[1])
    want = np.einsum("...ik,...kj->...ij", a.astype(np.float64), b.astype(np.float64))
    assert np.abs(res[1] - want).max() <= 700 * 2.0 ** -23 * np.abs(a).max() * np.abs(b).max() * 4


@pytest.mark.parametrize("m,n,k", [(130, 70, 300), (257, 129, 64), (33, 5, 1000)])
def test_cgemm_real_embedding_on_ffma(fg, oracle, m, n, k):
    """Plain CGEMM: with the FFMA kernel chosen for the embedded shape it runs
    as the real GEMM (M x 2K) x (2K x 2N); the 4M kernel otherwise."""
    r = rng(m + n + k)
    a = (r.standard_normal((m, k)) + 1j * r.standard_normal((m, k))).astype(np.complex64)
    b = (r.standard_normal((k, n)) + 1j * r.standard_normal((k, n))).astype(np.complex64)
    c0 = (r.standard_normal((m, n)) + 1j * r.standard_normal((m, n))).astype(np.complex64)
    exact = a.astype(np.complex128) @ b.astype(np.complex128)
    scale = np.linalg.norm(a.astype(np.complex128)) * np.linalg.norm(b.astype(np.complex128))
    for variant in (0, 4):
        with fg.tune_forced("f32", variant, 1):
            c = np.zeros((m, n), np.complex64)
            assert fg.gemm_c32(m, n, k, 1.0, 0.0, a, b, 0.0, 0.0, c)
            assert oracle.error_vs_dd(a, b, c) <= 2 * k * U32
            c = c0.copy()
            assert fg.gemm_c32(m, n, k, 0.5, 0.0, a, b, -1.0, 0.0, c)
            ref = 0.5 * exact - c0.astype(np.complex128)
            assert np.linalg.norm(c - ref) <= (2 * k + 4) * U32 * scale + 2 * U32 * np.linalg.norm(ref)


@pytest.mark.parametrize("splits", [1, 4])
@pytest.mark.parametrize("m,n,k", [(32, 600, 2000), (17, 300, 77), (70, 257, 500)])
def test_dmma_skinny_bit_identical(fg, m, n, k, splits):
    """f64 variant 5 (DMMA, 32 x 256 tiles of 32 x 32 warp tiles) runs the
    same m8n8k4 MMA sequence per output as variant 4: same bits."""
    r = rng(m * 7 + n + k)
    a = r.standard_normal((m, k))
    b = r.standard_normal((k, n))
    c0 = r.standard_normal((m, n))
    out = []
    for variant in (4, 5):
        with fg.tune_forced("f64", variant, splits):
            c = c0.copy()
            assert fg.gemm_f64(m, n, k, 0.75, a, b, -1.5, c)
            out.append(c)
    np.testing.assert_array_equal(out[0], out[1])
