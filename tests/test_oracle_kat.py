"""Known-answer tests that pin the CPU oracle (the reference ships no tests or
golden vectors; the Fortran cannot be built here).  They check the
restatement against properties the reference schemes must have:
polynomial exactness of the compact derivatives with their closures, the
filter transfer function, dense-LU agreement of the line solvers, and the
float32 rounding of the Gaussian coefficients."""
import numpy as np
import pytest

from conftest import rel_err
from shock_turbulence_b200.params import default_params

N = 32


@pytest.fixture(scope="module")
def orc(oracle_mod):
    return oracle_mod.Oracle(default_params(N, length=1.0))


def coord(d):
    x = np.linspace(0.0, 1.0, N)
    shp = [1, 1, 1]
    axis = {0: 0, 1: 2, 2: 1}[d]          # (Mx, Mz, My) C-order axes
    shp[axis] = N
    return np.broadcast_to(x.reshape(shp), (N, N, N)).copy()


@pytest.mark.parametrize("d", [0, 1, 2])
def test_first_derivative_exact_on_polynomials(orc, d):
    X = coord(d)
    F = np.ascontiguousarray(X ** 2)        # even about the symmetry plane
    dF = np.zeros_like(F)
    orc.dfd(d, 0, F, dF, 0, 1.0)
    assert np.abs(dF - 2 * X).max() < 1e-12
    F = np.ascontiguousarray(X ** 3)        # odd about the symmetry plane
    orc.dfd(d, 1, F, dF, 0, 1.0)
    assert np.abs(dF - 3 * X ** 2).max() < 1e-12
    # iadd/cadd semantics: dF += cadd * dF/dx
    dF2 = dF.copy()
    orc.dfd(d, 1, F, dF2, 1, -0.5)
    assert np.abs(dF2 - 0.5 * dF).max() < 1e-12


@pytest.mark.parametrize("d", [0, 1, 2])
def test_second_derivative_exact_on_polynomials(orc, d):
    X = coord(d)
    F = np.ascontiguousarray(X ** 2)
    dF, d2F = np.zeros_like(F), np.zeros_like(F)
    orc.d2fd2(d, 0, F, dF, d2F, 1)
    assert rel_err(d2F, 2.0 + 0 * X) < 1e-9      # closure rows cancel O(N^2) terms
    assert np.abs(dF - 2 * X).max() < 1e-12
    F = np.ascontiguousarray(X ** 3)
    orc.d2fd2(d, 1, F, dF, d2F, 0)
    assert rel_err(d2F, 6 * X) < 1e-9


def test_filter_transfer_function(orc):
    """Interior response: constants pass, the Nyquist mode is removed
    (Cook-Cabot eighth-order filter, src/LES_header:107-113)."""
    F = np.ones((N, N, N))
    F0 = np.zeros_like(F)
    orc.filter(1, 0, F, F0)
    assert np.abs(F0 - 1.0).max() < 1e-4        # boundary closures are not exact
    assert np.abs(F0[:, :, 4:-4] - 1.0).max() < 1e-13
    j = np.arange(N)
    F = np.ascontiguousarray(np.broadcast_to((-1.0) ** j, (N, N, N)))
    orc.filter(1, 0, F, F0)
    assert np.abs(F0[:, :, 8:-8]).max() < 1e-3


def test_gaussian_coefficients_are_float32(orc):
    """Gaussian_Filter interior weights are REAL*4 values: filtering a
    delta reproduces the float32-rounded coefficients exactly."""
    F = np.zeros((N, N, N))
    F[:, :, 16] = 1.0
    Fg = np.zeros_like(F)
    orc.gauss(1, F, Fg)
    expect = [np.float32(v) for v in (3565 / 10368, 3091 / 12960, 1997 / 25920, 149 / 12960,
                                      107 / 103680)]
    for k, e in enumerate(expect):
        assert Fg[0, 0, 16 + k] == float(e)
        assert Fg[0, 0, 16 - k] == float(e)


def _dense_tri(A, B, C, n):
    M = np.zeros((n, n))
    for i in range(n):
        M[i, i] = B[i]
        if i > 0:
            M[i, i - 1] = A[i]
        if i < n - 1:
            M[i, i + 1] = C[i]
    return M


@pytest.mark.parametrize("nper", [0, 1])
def test_tridiagonal_matches_dense(oracle_mod, nper):
    rng = np.random.default_rng(0)
    n, lot = 24, 7
    A = rng.uniform(0.1, 0.4, (n, lot)); C = rng.uniform(0.1, 0.4, (n, lot)); B = np.ones((n, lot))
    R = rng.normal(size=(n, lot))
    X = R.copy()
    oracle_mod.tridiagonal(A, B, C, X, nper)
    for L in range(lot):
        M = _dense_tri(A[:, L], B[:, L], C[:, L], n)
        if nper:
            M[0, n - 1] = A[0, L]
            M[n - 1, 0] = C[n - 1, L]
        assert rel_err(X[:, L], np.linalg.solve(M, R[:, L])) < 1e-13


@pytest.mark.parametrize("nper", [0, 1])
def test_pentadiagonal_matches_dense(oracle_mod, nper):
    rng = np.random.default_rng(1)
    n, lot = 20, 5
    A, B, D, E = (rng.uniform(0.05, 0.2, (n, lot)) for _ in range(4))
    C = np.ones((n, lot))
    R = rng.normal(size=(n, lot))
    X = R.copy()
    oracle_mod.pentadiagonal(A, B, C, D, E, X, nper)
    for L in range(lot):
        M = np.zeros((n, n))
        for i in range(n):
            for off, arr in ((-2, A), (-1, B), (0, C), (1, D), (2, E)):
                j = i + off
                if 0 <= j < n:
                    M[i, j] = arr[i, L]
                elif nper:
                    M[i, j % n] = arr[i, L]
        assert rel_err(X[:, L], np.linalg.solve(M, R[:, L])) < 1e-12


def test_filter_matches_dense_solve(orc):
    """The filter's pentadiagonal solve equals a dense solve of its LHS."""
    rng = np.random.default_rng(2)
    F = rng.normal(size=(N, N, N))
    F0 = np.zeros_like(F)
    orc.filter(1, 0, F, F0)
    a, b, al, ab = 6.6624e-01, 1.6688e-01, 0.45, 0.45
    M = np.zeros((N, N))
    for i in range(N):
        M[i, max(0, i - 2):i + 3] = [b, a, 1, a, b][max(0, 2 - i):5 - max(0, i + 3 - N)]
    M[0, :] = 0; M[0, 0] = 1; M[0, 1] = 2 * a; M[0, 2] = 2 * b
    M[1, :] = 0; M[1, 0] = a; M[1, 1] = 1 + b; M[1, 2] = a; M[1, 3] = b
    M[N - 1, :] = 0; M[N - 1, N - 1] = 1
    for r in (N - 2, N - 3):
        M[r, :] = 0; M[r, r - 1] = al; M[r, r] = 1; M[r, r + 1] = ab
    line = F0[3, 5, :]
    W = M @ line                                   # reconstruct the explicit RHS
    Wn = np.linalg.solve(M, W)
    assert rel_err(Wn, line) < 1e-11
