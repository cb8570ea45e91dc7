"""multi_dot and matrix_power on device-resident operands against the
restated reference (same product order), within the chained GEMM bound."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

U64, U32 = 2.0 ** -53, 2.0 ** -24


@pytest.mark.parametrize("dt,u", [(np.float64, U64), (np.float32, U32)])
@pytest.mark.parametrize("dims", [[30, 400, 5, 300], [7, 200, 200, 3, 150, 60], [300, 300, 300, 300, 300]])
def test_multi_dot(fg, oracle, dt, u, dims):
    rng = np.random.default_rng(sum(dims))
    mats = [rng.uniform(-1, 1, (dims[i], dims[i + 1])).astype(dt) for i in range(len(dims) - 1)]
    got = fg.multi_dot([fg.DeviceArray.from_numpy(x) for x in mats]).to_numpy()
    want = oracle.multi_dot(mats)
    exact = mats[0].astype(np.float64)
    for x in mats[1:]:
        exact = exact @ x.astype(np.float64)
    scale = np.prod([np.linalg.norm(x.astype(np.float64)) for x in mats])
    kk = sum(dims)
    assert np.linalg.norm(got - exact) / scale <= kk * u
    assert np.linalg.norm(got - exact) <= 2 * np.linalg.norm(want - exact) + kk * u * scale


def test_multi_dot_vector_ends_and_errors(fg):
    rng = np.random.default_rng(1)
    v = rng.standard_normal(50)
    a = rng.standard_normal((50, 40))
    b = rng.standard_normal((40, 30))
    w = rng.standard_normal(30)
    dv, da, db, dw = (fg.DeviceArray.from_numpy(x) for x in (v, a, b, w))
    got = fg.multi_dot([dv, da, db, dw]).to_numpy()
    assert got.shape == ()
    np.testing.assert_allclose(got, v @ a @ b @ w, rtol=1e-12, atol=1e-12)
    with pytest.raises(fg.ShapeMismatch):
        fg.multi_dot([da, da, db])
    with pytest.raises(fg.InvalidValue):
        fg.multi_dot([da])


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("p", [0, 1, 2, 3, 7, 10])
def test_matrix_power(fg, oracle, dt, p):
    rng = np.random.default_rng(p)
    n = 64
    a = (rng.uniform(-1, 1, (n, n)) / np.sqrt(n)).astype(dt)
    got = fg.matrix_power(fg.DeviceArray.from_numpy(a), p).to_numpy()
    want = oracle.matrix_power(a, p)
    exact = np.linalg.matrix_power(a.astype(np.float64), p)
    tol = (1e-12 if dt == np.float64 else 1e-4) * max(1, p)
    assert np.max(np.abs(got - exact)) <= tol
    assert np.max(np.abs(got - exact)) <= 2 * np.max(np.abs(want - exact)) + tol / 10


def test_matrix_power_errors(fg):
    a = fg.DeviceArray.from_numpy(np.eye(3))
    with pytest.raises(fg.Unsupported):
        fg.matrix_power(a, -1)
    with pytest.raises(fg.ShapeMismatch):
        fg.matrix_power(fg.DeviceArray.from_numpy(np.zeros((2, 3))), 2)


@pytest.mark.parametrize("dt,u", [(np.float64, U64), (np.float32, U32), (np.complex128, U64)])
@pytest.mark.parametrize("sa,sb,axes", [
    ((3, 4, 5), (4, 5, 6), 2),                 # identity permutations
    ((3, 4, 5), (5, 4, 2), ([1, 2], [1, 0])),  # both permuted
    ((6, 7, 8, 9), (9, 7, 5), ([3, 1], [0, 1])),
    ((30, 40), (40, 50), 1),
    ((5, 6), (7, 8), 0),                       # outer product
    ((4, 5), (5, 4), ([0, 1], [1, 0])),        # full contraction -> shape ()
])
def test_tensordot(fg, oracle, dt, u, sa, sb, axes):
    rng = np.random.default_rng(len(sa) * 10 + len(sb))
    a = rng.standard_normal(sa)
    b = rng.standard_normal(sb)
    if dt == np.complex128:
        a = a + 1j * rng.standard_normal(sa)
        b = b + 1j * rng.standard_normal(sb)
    a, b = a.astype(dt), b.astype(dt)
    got = fg.tensordot(fg.DeviceArray.from_numpy(a), fg.DeviceArray.from_numpy(b), axes).to_numpy()
    if isinstance(axes, int):
        ax = (list(range(a.ndim - axes, a.ndim)), list(range(axes)))
    else:
        ax = axes
    want = np.tensordot(a.astype(np.complex128), b.astype(np.complex128), axes=ax)
    assert got.shape == want.shape
    k = max(1, int(np.prod([a.shape[i] for i in ax[0]])))
    scale = np.linalg.norm(a) * np.linalg.norm(b)
    assert np.linalg.norm(got - want) <= 4 * k * u * scale + 1e-300
    if dt == np.float64:
        ref = oracle.tensordot(a, b, ax[0], ax[1])
        assert np.linalg.norm(got - want) <= 2 * np.linalg.norm(ref - want) + 2 * k * u * scale


def test_tensordot_errors(fg):
    a = fg.DeviceArray.from_numpy(np.zeros((3, 4)))
    b = fg.DeviceArray.from_numpy(np.zeros((5, 6)))
    with pytest.raises(fg.ShapeMismatch):
        fg.tensordot(a, b, 1)
    with pytest.raises(fg.ShapeMismatch):
        fg.tensordot(a, b, ([0], [0, 1]))


@pytest.mark.parametrize("spec,sa,sb", [
    ("ij,jk->ik", (30, 40), (40, 20)),          # the reference's matmul shortcut
    ("ij,jk", (30, 40), (40, 20)),              # implicit output
    ("bij,bjk->bik", (4, 30, 40), (4, 40, 20)),  # batched
    ("ij,kj->ik", (30, 40), (20, 40)),          # B transposed
    ("ijk,kjl->il", (5, 6, 7), (7, 6, 8)),      # two contracted labels, permuted
    ("bij,bjk->kib", (3, 5, 6), (3, 6, 4)),     # output permuted
    ("i,j->ij", (7,), (9,)),                    # outer product
    ("ij,ij->", (6, 5), (6, 5)),                # full contraction
])
def test_einsum_pairwise(fg, spec, sa, sb):
    rng = np.random.default_rng(len(spec))
    a = rng.standard_normal(sa)
    b = rng.standard_normal(sb)
    got = fg.einsum(spec, fg.DeviceArray.from_numpy(a), fg.DeviceArray.from_numpy(b)).to_numpy()
    want = np.einsum(spec, a, b)
    assert got.shape == want.shape
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12 * max(1.0, np.abs(want).max()))


def test_einsum_unsupported_forms(fg):
    a = fg.DeviceArray.from_numpy(np.zeros((3, 3)))
    with pytest.raises(fg.Unsupported):
        fg.einsum("ii,ij->j", a, a)   # repeated label within an operand (trace)
    with pytest.raises(fg.ShapeMismatch):
        fg.einsum("ij,jk->ik", a, fg.DeviceArray.from_numpy(np.zeros((4, 2))))
