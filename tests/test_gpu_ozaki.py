"""GPU tests of the split (INT8 Ozaki) DGEMM / ZGEMM against the
double-double oracle: the default form (scheme II, 16 moduli; its own
file covers other moduli counts) and scheme I with explicit slice counts.

Tolerances (normwise ||C - C_ref||_F / (||A||_F ||B||_F)):
* default (9 slices), every case: K * 2^-53, the deterministic bound a plain
  FP64 GEMM meets, plus (S+2) * 2^(2-7S) for the digit truncation and the
  dropped slice pairs (which matters only for tiny K);
* default slices, operands built as diag(10^(s u)) G diag(10^(s v)) with
  spread s in {0, 4, 8}: no worse than 2x the plain FP64 kernel's error on the
  same operands, plus a floor of 2^-60 for cases where both are near exact;
* fewer slices: the representation bound K * 2^(6 - 7S) (digit truncation
  below 2^-7S of the balanced row / column maxima).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

U64 = 2.0 ** -53


def spread_operands(rng, m, k, n, s):
    """A = diag(10^(s u)) G diag(10^(s v)) (the split-DGEMM benchmark family)."""
    def one(r, c):
        g = rng.standard_normal((r, c))
        u = rng.uniform(-1, 1, r)
        v = rng.uniform(-1, 1, c)
        return (10.0 ** (s * u))[:, None] * g * (10.0 ** (s * v))[None, :]
    return one(m, k), one(k, n)


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (17, 13, 9), (128, 256, 128), (300, 257, 129),
                                   (513, 257, 300), (1024, 1024, 1024)])
def test_f64_split_bound(fg, oracle, m, n, k):
    rng = np.random.default_rng(m + 3 * n + 7 * k)
    a = rng.uniform(-1, 1, (m, k))
    b = rng.uniform(-1, 1, (k, n))
    c = np.zeros((m, n))
    assert fg.gemm_f64(m, n, k, 1.0, a, b, 0.0, c, mode="split")
    err = oracle.error_vs_dd(a, b, c)
    assert err <= k * U64 + 11 * 2.0 ** (2 - 63), err


@pytest.mark.parametrize("slices", [0, 9])
@pytest.mark.parametrize("spread", [0, 4, 8])
def test_f64_split_vs_plain_per_spread(fg, oracle, spread, slices):
    rng = np.random.default_rng(100 + spread)
    m = n = k = 768
    a, b = spread_operands(rng, m, k, n, spread)
    cs, cp = np.zeros((m, n)), np.zeros((m, n))
    assert fg.gemm_f64(m, n, k, 1.0, a, b, 0.0, cs, mode="split", ozaki_slices=slices)
    assert fg.gemm_f64(m, n, k, 1.0, a, b, 0.0, cp, mode="plain")
    es = oracle.error_vs_dd(a, b, cs)
    ep = oracle.error_vs_dd(a, b, cp)
    assert es <= 2 * ep + 2.0 ** -60, (spread, es, ep)


@pytest.mark.parametrize("slices", [4, 5, 6, 7])
def test_f64_split_fewer_slices(fg, oracle, slices):
    rng = np.random.default_rng(slices)
    m, n, k = 200, 180, 333
    a = rng.standard_normal((m, k))
    b = rng.standard_normal((k, n))
    c = np.zeros((m, n))
    assert fg.gemm_f64(m, n, k, 1.0, a, b, 0.0, c, mode="split", ozaki_slices=slices)
    err = oracle.error_vs_dd(a, b, c)
    assert err <= max(k * U64, k * 2.0 ** (6 - 7 * slices)), err


def test_f64_split_alpha_beta(fg):
    rng = np.random.default_rng(5)
    m, n, k = 150, 260, 190
    a, b = rng.uniform(-1, 1, (m, k)), rng.uniform(-1, 1, (k, n))
    c0 = rng.uniform(-1, 1, (m, n))
    c = c0.copy()
    assert fg.gemm_f64(m, n, k, -0.75, a, b, 1.5, c, mode="split")
    want = -0.75 * (a @ b) + 1.5 * c0
    assert np.max(np.abs(c - want)) < 1e-12


def test_f64_split_nonfinite_rows_and_zero_rows(fg):
    rng = np.random.default_rng(6)
    m, n, k = 40, 50, 60
    a, b = rng.uniform(-1, 1, (m, k)), rng.uniform(-1, 1, (k, n))
    a[3, 7] = np.nan
    a[5, :] = 0.0
    c = np.zeros((m, n))
    assert fg.gemm_f64(m, n, k, 1.0, a, b, 0.0, c, mode="split")
    assert np.all(np.isnan(c[3]))
    assert np.all(c[5] == 0.0)
    ok = [i for i in range(m) if i != 3]
    assert np.max(np.abs(c[ok] - (a[ok] @ b))) < 1e-13


@pytest.mark.parametrize("m,n,k", [(17, 13, 9), (128, 96, 200), (257, 129, 300)])
def test_c64_split(fg, oracle, m, n, k):
    rng = np.random.default_rng(k)
    a = rng.standard_normal((m, k)) + 1j * rng.standard_normal((m, k))
    b = rng.standard_normal((k, n)) + 1j * rng.standard_normal((k, n))
    cs = np.zeros((m, n), np.complex128)
    cp = np.zeros((m, n), np.complex128)
    assert fg.gemm_c64(m, n, k, 1.0, 0.0, a, b, 0.0, 0.0, cs, mode="split")
    assert fg.gemm_c64(m, n, k, 1.0, 0.0, a, b, 0.0, 0.0, cp)
    es = oracle.error_vs_dd(a, b, cs)
    ep = oracle.error_vs_dd(a, b, cp)
    assert es <= 2 * k * U64, es
    assert es <= 2 * ep + 2.0 ** -60, (es, ep)


def test_split_matmul_batched_f64(fg):
    rng = np.random.default_rng(9)
    a = rng.standard_normal((3, 40, 70))
    b = rng.standard_normal((70, 30))
    got = fg.matmul(a, b, mode="split")
    want = np.matmul(a, b)
    assert np.max(np.abs(got - want)) < 1e-12


@pytest.mark.parametrize("m,n,k,cplx", [(64, 48, 15000, False), (40, 24, 7600, True)])
def test_split_long_k_group_pieces(fg, oracle, m, n, k, cplx):
    # scheme I, 9 slices: the top slice group's concatenated K (9 x K, x2
    # embedded for complex) exceeds what one int32 accumulator holds exactly,
    # so that group runs as several launches; the result keeps the 9-slice
    # bound.
    rng = np.random.default_rng(k)
    a = rng.uniform(-1, 1, (m, k))
    b = rng.uniform(-1, 1, (k, n))
    if cplx:
        a = a + 1j * rng.uniform(-1, 1, (m, k))
        b = b + 1j * rng.uniform(-1, 1, (k, n))
        c = np.zeros((m, n), np.complex128)
        assert fg.gemm_c64(m, n, k, 1.0, 0.0, a, b, 0.0, 0.0, c, mode="split", ozaki_slices=9)
    else:
        c = np.zeros((m, n))
        assert fg.gemm_f64(m, n, k, 1.0, a, b, 0.0, c, mode="split", ozaki_slices=9)
    err = oracle.error_vs_dd(a, b, c)
    assert err <= (2 if cplx else 1) * k * U64 + 11 * 2.0 ** (2 - 63), err


_PER_GROUP_SCRIPT = r"""
import sys, numpy as np
sys.path.insert(0, sys.argv[1])
import ferray_b200 as fg
d = np.load(sys.argv[2])
a, b, cplx = d["a"], d["b"], bool(d["cplx"])
m, k = a.shape
n = b.shape[1]
c = np.zeros((m, n), a.dtype)
sl = int(d["slices"])
if cplx:
    assert fg.gemm_c64(m, n, k, 1.5, 0.0, a, b, 0.0, 0.0, c, mode="split", ozaki_slices=sl)
else:
    assert fg.gemm_f64(m, n, k, 1.5, a, b, 0.0, c, mode="split", ozaki_slices=sl)
np.save(sys.argv[3], c)
"""


@pytest.mark.parametrize("slices", [9, 16])
@pytest.mark.parametrize("m,n,k,cplx", [(300, 257, 129, False), (513, 1000, 700, False), (200, 150, 300, True)])
def test_fused_groups_bit_identical_to_group_launches(fg, tmp_path, m, n, k, cplx, slices):
    """All slice groups (scheme I) or all moduli (scheme II) in one launch,
    the default, give the same bits as one launch per group / modulus
    (FG_OZAKI_FUSED=0, run in a child process): scheme I's FP64 epilogue adds
    the groups to C in the same order either way, and scheme II's residue
    bytes do not depend on the launch."""
    import os
    import subprocess
    import sys
    r = np.random.default_rng(m + n + k)
    a = r.standard_normal((m, k)) * 10.0 ** r.uniform(-4, 4, (m, 1))
    b = r.standard_normal((k, n)) * 10.0 ** r.uniform(-4, 4, (1, n))
    if cplx:
        a = a + 1j * r.standard_normal((m, k))
        b = b + 1j * r.standard_normal((k, n))
    c = np.zeros((m, n), a.dtype)
    if cplx:
        assert fg.gemm_c64(m, n, k, 1.5, 0.0, a, b, 0.0, 0.0, c, mode="split", ozaki_slices=slices)
    else:
        assert fg.gemm_f64(m, n, k, 1.5, a, b, 0.0, c, mode="split", ozaki_slices=slices)
    np.savez(tmp_path / "in.npz", a=a, b=b, cplx=cplx, slices=slices)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, FG_OZAKI_FUSED="0")
    subprocess.run([sys.executable, "-c", _PER_GROUP_SCRIPT, root, str(tmp_path / "in.npz"),
                    str(tmp_path / "out.npy")], check=True, env=env, timeout=300)
    ref = np.load(tmp_path / "out.npy")
    assert np.array_equal(c.view(np.uint8), ref.view(np.uint8))
