"""st_tridiagonal_noalloc: the allocation-free tridiagonal entry point agrees
with st_tridiagonal and with the CPU oracle's tridiagonal, call after call,
and rejects what it cannot serve.

Kept in its own file, collected last, so that it also runs after every other
GPU test in the same process; it passes alone in a fresh process as well."""
import ctypes

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-12
LIMIT = 1 << 18          # n*lot limit of st_tridiagonal_noalloc
ST_E_ARG = -1


@pytest.fixture(scope="module")
def solver():
    from shock_turbulence_b200 import Solver, default_params
    return Solver(default_params(32))


def _system(rng, n, lot):
    A = rng.uniform(0.1, 0.4, (n, lot))
    C = rng.uniform(0.1, 0.4, (n, lot))
    B = rng.uniform(0.9, 1.1, (n, lot))
    R = rng.normal(size=(n, lot))
    return A, B, C, R


def _noalloc(s, A, B, C, R, n, lot, nper):
    return s.lib.st_tridiagonal_noalloc(s._h, A.data_ptr(), B.data_ptr(), C.data_ptr(), R.data_ptr(),
                                        n, lot, nper)


@pytest.mark.parametrize("nper", [0, 1])
def test_two_calls_match_st_tridiagonal(solver, oracle_mod, nper):
    import torch
    rng = np.random.default_rng(11 + nper)
    for n, lot in ((40, 300), (512, 512)):          # the second size is exactly at the limit
        for _ in range(2):                           # two calls in a row reuse the scratch
            A, B, C, R = _system(rng, n, lot)
            ref = R.copy()
            solver.tridiagonal(A, B, C, ref, n, lot, nper)
            dA, dB, dC, dR = (torch.from_numpy(x).cuda() for x in (A, B, C, R))
            st = _noalloc(solver, dA, dB, dC, dR, n, lot, nper)
            assert st == 0, solver.lib.st_last_error(solver._h)
            assert rel_err(dR.cpu().numpy(), ref) < TOL
            orc = R.copy()
            oracle_mod.tridiagonal(A.copy(), B.copy(), C.copy(), orc, nper)
            assert rel_err(dR.cpu().numpy(), orc) < TOL
            # the coefficients are inputs only
            assert torch.equal(dA.cpu(), torch.from_numpy(A))
            assert torch.equal(dB.cpu(), torch.from_numpy(B))


@pytest.mark.parametrize("nper", [0, 1])
@pytest.mark.parametrize("n", [1, 2, 3, 5])
def test_short_lines_match_the_oracle(solver, oracle_mod, nper, n):
    """The solver's special cases of very short (periodic) lines."""
    import torch
    rng = np.random.default_rng(100 * n + nper)
    lot = 64
    for _ in range(2):
        A, B, C, R = _system(rng, n, lot)
        orc = R.copy()
        oracle_mod.tridiagonal(A.copy(), B.copy(), C.copy(), orc, nper)
        dA, dB, dC, dR = (torch.from_numpy(x).cuda() for x in (A, B, C, R))
        st = _noalloc(solver, dA, dB, dC, dR, n, lot, nper)
        assert st == 0, solver.lib.st_last_error(solver._h)
        assert rel_err(dR.cpu().numpy(), orc) < TOL


def test_rejects_sizes_beyond_the_limit(solver):
    import torch
    n, lot = 513, 512
    assert n * lot > LIMIT
    A, B, C, R = (torch.ones((n, lot), dtype=torch.float64, device="cuda") for _ in range(4))
    st = _noalloc(solver, A, B, C, R, n, lot, 0)
    assert st == ST_E_ARG
    assert b"exceeds the limit" in solver.lib.st_last_error(solver._h)
    assert torch.all(R == 1.0)


def test_rejects_host_arrays(solver):
    n, lot = 16, 8
    A, B, C, R = (np.ones((n, lot)) for _ in range(4))
    p = [x.ctypes.data_as(ctypes.c_void_p) for x in (A, B, C, R)]
    st = solver.lib.st_tridiagonal_noalloc(solver._h, *p, n, lot, 0)
    assert st == ST_E_ARG
    assert b"device arrays" in solver.lib.st_last_error(solver._h)
    assert np.all(R == 1.0)
