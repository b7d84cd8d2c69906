"""Host-side format logic: the seeded generator, the CSC assembly and the
device layout.  CPU only."""
import numpy as np

from bbjd_b200.pencils import make_pencil, start_vector


def test_generator_is_deterministic():
    a = make_pencil(8, 16, 4, seed=0)
    b = make_pencil(8, 16, 4, seed=0)
    c = make_pencil(8, 16, 4, seed=1)
    for f in ("Ad", "Al", "Au", "E", "F", "Bd"):
        assert np.array_equal(getattr(a, f), getattr(b, f))
    assert not np.array_equal(a.Ad, c.Ad)
    assert np.array_equal(start_vector(100, 1), start_vector(100, 1))


def test_generator_law():
    P = make_pencil(16, 64, 8, seed=0)
    assert np.all(P.Al[0] == 0) and np.all(P.Au[-1] == 0)
    shifts = 1j * np.linspace(-50, 50, 64) + np.linspace(0, 10, 64)
    diag = np.einsum("jii->ji", P.Ad)
    # the noise on the diagonal is O(1/sqrt(b)); the shift dominates
    assert np.abs(diag.mean(axis=1) - shifts).max() < 1.0
    assert np.all(np.abs(np.einsum("jii->ji", P.Bd) - 1) < 1.0)


def test_csc_matches_block_products():
    P = make_pencil(8, 32, 4, seed=2)
    A, B = P.to_csc("A"), P.to_csc("B")
    rng = np.random.default_rng(7)
    x = rng.standard_normal(P.n) + 1j * rng.standard_normal(P.n)
    assert np.allclose(A @ x, P.matvec_A(x), atol=1e-13)
    assert np.allclose(B @ x, P.matvec_B(x), atol=1e-13)
    assert A.nnz == 3 * 32 * 64 - 2 * 64 + 2 * 256 * 4 + 4 * 4
    # B's tau rows are zero: B is singular
    assert np.all((B @ x)[P.nb:] == 0)


def test_device_layout_is_column_major():
    P = make_pencil(8, 4, 2, seed=0)
    d = P.device_arrays()
    j, i, c = 2, 3, 5
    assert d["Ad"].reshape(-1)[j * 64 + c * 8 + i] == P.Ad[j, i, c]
    assert d["E"][1 * P.nb + 7] == P.E[7, 1]
    assert d["FT"][9 * 2 + 1] == P.F[1, 9]
    # flat and contiguous: a reshape or a float64 view keeps the order
    for name, a in d.items():
        assert a.ndim == 1 and a.flags.c_contiguous, name
        np.testing.assert_array_equal(a.reshape(-1).view(np.float64).view(np.complex128), a)


def test_shifted_pencil():
    P = make_pencil(8, 8, 2, seed=0)
    S = P.shifted(3.0)
    rng = np.random.default_rng(1)
    x = rng.standard_normal(P.n) + 0j
    assert np.allclose(S.matvec_A(x), P.matvec_A(x) - 3.0 * P.matvec_B(x))
