"""GPU tests of Ozaki scheme II (ozaki_slices 12..20: that many pairwise
coprime moduli <= 256, one int8 GEMM per modulus on symmetric residues,
the product rebuilt by the Chinese remainder theorem) against the
double-double oracle.

The integer operands carry P bits below each balanced row / column maximum,
P = min(59, floor((floor(log2 Mp) - ceil(log2 K) - 2) / 2)) for the moduli product
Mp; entries within 2^(53 - P) of their row maximum are exact.  Tolerances
(normwise ||C - C_ref||_F / (||A||_F ||B||_F)):
* 16 or more moduli (P >= 55 up to K = 8192): no worse than 2x the plain
  FP64 kernel's error on the same operands, per exponent spread 0, 4, 8,
  plus a floor of 2^-60;
* 12 moduli (P about 43): K 2^(4 - P), the rounding bound of the operands.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

U64 = 2.0 ** -53
MODULI = [256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197, 193, 191, 181, 179, 173]


def precision_bits(n, k):
    mp = 1
    for m in MODULI[:n]:
        mp *= m
    logk = 0
    while (1 << logk) < k:
        logk += 1
    return min(59, (mp.bit_length() - 1 - logk - 2) // 2)


def spread_operands(rng, m, k, n, s, cplx=False):
    def one(r, c):
        g = rng.standard_normal((r, c))
        if cplx:
            g = g + 1j * rng.standard_normal((r, c))
        u = rng.uniform(-1, 1, r)
        v = rng.uniform(-1, 1, c)
        return (10.0 ** (s * u))[:, None] * g * (10.0 ** (s * v))[None, :]
    return one(m, k), one(k, n)


@pytest.mark.parametrize("moduli", [16, 17, 20])
@pytest.mark.parametrize("spread", [0, 4, 8])
def test_scheme2_vs_plain_per_spread(fg, oracle, moduli, spread):
    rng = np.random.default_rng(200 + spread + moduli)
    m, n, k = 700, 520, 900
    a, b = spread_operands(rng, m, k, n, spread)
    c2, cp = np.zeros((m, n)), np.zeros((m, n))
    assert fg.gemm_f64(m, n, k, 1.0, a, b, 0.0, c2, mode="split", ozaki_slices=moduli)
    assert fg.gemm_f64(m, n, k, 1.0, a, b, 0.0, cp)
    e2, ep = oracle.error_vs_dd(a, b, c2), oracle.error_vs_dd(a, b, cp)
    assert e2 <= 2 * ep + 2.0 ** -60, (moduli, spread, e2, ep)


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (17, 13, 9), (128, 256, 128), (300, 257, 129),
                                   (513, 257, 300), (64, 40, 20000)])
def test_scheme2_bound(fg, oracle, m, n, k):
    rng = np.random.default_rng(m + n + k)
    a = rng.uniform(-1, 1, (m, k))
    b = rng.uniform(-1, 1, (k, n))
    for moduli in (12, 17):
        c = np.zeros((m, n))
        assert fg.gemm_f64(m, n, k, 1.0, a, b, 0.0, c, mode="split", ozaki_slices=moduli)
        err = oracle.error_vs_dd(a, b, c)
        p = precision_bits(moduli, k)
        assert err <= k * U64 + k * 2.0 ** (4 - p), (moduli, err)


@pytest.mark.parametrize("spread", [0, 8])
def test_scheme2_complex(fg, oracle, spread):
    rng = np.random.default_rng(300 + spread)
    m, n, k = 260, 190, 330
    a, b = spread_operands(rng, m, k, n, spread, cplx=True)
    c2 = np.zeros((m, n), np.complex128)
    cp = np.zeros((m, n), np.complex128)
    assert fg.gemm_c64(m, n, k, 1.0, 0.0, a, b, 0.0, 0.0, c2, mode="split", ozaki_slices=17)
    assert fg.gemm_c64(m, n, k, 1.0, 0.0, a, b, 0.0, 0.0, cp)
    e2, ep = oracle.error_vs_dd(a, b, c2), oracle.error_vs_dd(a, b, cp)
    assert e2 <= 2 * ep + 2.0 ** -60, (e2, ep)


def test_scheme2_alpha_beta_nonfinite_and_zero_rows(fg):
    rng = np.random.default_rng(7)
    m, n, k = 150, 260, 190
    a, b = rng.uniform(-1, 1, (m, k)), rng.uniform(-1, 1, (k, n))
    c0 = rng.uniform(-1, 1, (m, n))
    c = c0.copy()
    assert fg.gemm_f64(m, n, k, -0.75, a, b, 1.5, c, mode="split", ozaki_slices=17)
    assert np.max(np.abs(c - (-0.75 * (a @ b) + 1.5 * c0))) < 1e-12
    a[3, 7] = np.nan
    a[5, :] = 0.0
    c = np.zeros((m, n))
    assert fg.gemm_f64(m, n, k, 1.0, a, b, 0.0, c, mode="split", ozaki_slices=17)
    assert np.all(np.isnan(c[3]))
    assert np.all(c[5] == 0.0)
    ok = [i for i in range(m) if i != 3]
    assert np.max(np.abs(c[ok] - (a[ok] @ b))) < 1e-13


def test_scheme2_rejects_bad_counts(fg):
    from ferray_b200 import _lib as L
    a, b, c = np.ones((4, 4)), np.ones((4, 4)), np.zeros((4, 4))
    for bad in (11, 21):
        with pytest.raises(fg.FerrayError):
            fg.gemm_f64(4, 4, 4, 1.0, a, b, 0.0, c, mode="split", ozaki_slices=bad)
