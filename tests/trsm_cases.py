"""The reference's TRSM test cases (ferray-linalg/src/trsm.rs:520-712),
restated: (name, dtype, upper, unit_diag, m, n, alpha, b generator,
residual tolerance).  Each case checks op(A) X against alpha B."""
import numpy as np

import oracle

CASES = [
    # trsm.rs:520-541
    ("lln_f64_small", np.float64, False, False, 5, 3, 1.0, lambda i: i * 0.7 + 1.0, 1e-10),
    # trsm.rs:543-565 (m > 32: recursion and trailing update)
    ("lln_f64_large_blocked", np.float64, False, False, 80, 7, 1.0, lambda i: np.sin(i * 0.13) + 1.0, 1e-9),
    # trsm.rs:593-613
    ("lun_f64_small", np.float64, True, False, 5, 3, 1.0, lambda i: i * 0.7 + 1.0, 1e-10),
    # trsm.rs:615-635
    ("lun_f64_large_blocked", np.float64, True, False, 100, 5, 1.0, lambda i: np.cos(i * 0.17), 1e-9),
    # trsm.rs:637-659
    ("alpha_scales_b", np.float64, False, False, 4, 2, 3.0, lambda i: i + 1.0, 1e-10),
    # trsm.rs:661-686
    ("lln_f32_blocked", np.float32, False, False, 65, 4, 1.0, lambda i: i * 0.13 + 0.5, 1e-3),
    # trsm.rs:688-712
    ("lun_f32_blocked", np.float32, True, False, 70, 3, 1.0, lambda i: i * 0.07 - 0.5, 1e-3),
]


def operands(case):
    _, dt, upper, _, m, n, _, gen, _ = case
    a = oracle.trsm_test_triangle(m, upper).astype(dt)
    b = gen(np.arange(m * n, dtype=np.float64)).astype(dt).reshape(m, n)
    return a, b


def residual_ok(case, a, b, x):
    """max |A X - alpha B| within the case's tolerance (the reference
    computes A X with a naive loop; float64 here)."""
    alpha, tol = case[6], case[8]
    r = a.astype(np.float64) @ x.astype(np.float64) - alpha * b.astype(np.float64)
    return float(np.abs(r).max()) < tol


def unit_diag_triangle(m=6):
    """trsm.rs:567-591: the lower test triangle with its diagonal set to 1,
    solved with unit_diag true and false (results must agree)."""
    a = oracle.trsm_test_triangle(m, False)
    a[np.arange(m), np.arange(m)] = 1.0
    return a


def random_triangle(m, dtype, upper, seed):
    """Well-conditioned random triangle for large cases: off-diagonal
    U[-1, 1) / m, diagonal U[1, 2)."""
    r = np.random.default_rng(seed)
    a = r.uniform(-1.0, 1.0, (m, m)) / m
    a[np.arange(m), np.arange(m)] = r.uniform(1.0, 2.0, m)
    a = np.triu(a) if upper else np.tril(a)
    return a.astype(dtype)
