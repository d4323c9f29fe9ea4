"""GPU parity of the line operators against the CPU oracle, through the C ABI
(host arrays and device tensors).  Tolerance: 1e-12 normwise relative per
derivative / filter call (max|gpu-oracle| / max|oracle|)."""
import numpy as np
import pytest

from conftest import rel_err
from shock_turbulence_b200.params import default_params

pytestmark = pytest.mark.gpu
TOL = 1e-12
GRIDS = [(64, 64, 64), (64, 96, 32)]        # (nx, ny, nz); the second checks the axis mapping


@pytest.fixture(scope="module", params=GRIDS, ids=lambda g: "x".join(map(str, g)))
def pair(request, oracle_mod):
    from shock_turbulence_b200 import Solver
    nx, ny, nz = request.param
    p = default_params(nx, ny, nz, length=2.0)
    p.y_leng, p.z_leng = 3.0, 1.5
    return Solver(p), oracle_mod.Oracle(p)


def field(s, seed, smooth=True):
    rng = np.random.default_rng(seed)
    nx, nz, ny = s.shape
    f = rng.normal(size=s.shape)
    if smooth:
        x = np.linspace(0, 1, nx)[:, None, None]
        z = np.linspace(0, 1, nz)[None, :, None]
        y = np.linspace(0, 1, ny)[None, None, :]
        f = np.sin(3 * x + 1) * np.cos(2 * y) * np.exp(z) + 0.05 * f
    return np.ascontiguousarray(f)


DIRS = ["X", "Y", "Z"]


@pytest.mark.parametrize("d", [0, 1, 2])
@pytest.mark.parametrize("asym", [0, 1])
@pytest.mark.parametrize("iadd,cadd", [(0, 1.0), (1, -0.5)])
def test_first_derivative(pair, d, asym, iadd, cadd):
    s, o = pair
    F = field(s, 10 + d)
    base = field(s, 20, smooth=False)
    g, r = base.copy(), base.copy()
    getattr(s, f"DFD{DIRS[d]}_{'asym' if asym else 'sym'}")(F, g, iadd, cadd)
    o.dfd(d, asym, F, r, iadd, cadd)
    assert rel_err(g, r) < TOL


@pytest.mark.parametrize("d", [0, 1, 2])
@pytest.mark.parametrize("asym", [0, 1])
def test_second_derivative(pair, d, asym):
    s, o = pair
    F = field(s, 30 + d)
    g1, g2, r1, r2 = (np.zeros(s.shape) for _ in range(4))
    getattr(s, f"D2FD{DIRS[d]}2_{'asym' if asym else 'sym'}")(F, g1, g2, 1)
    o.d2fd2(d, asym, F, r1, r2, 1)
    assert rel_err(g2, r2) < TOL
    assert rel_err(g1, r1) < TOL


@pytest.mark.parametrize("d", [0, 1, 2])
@pytest.mark.parametrize("asym", [0, 1])
def test_compact_filter_direction(pair, d, asym):
    s, o = pair
    F = field(s, 40 + d, smooth=False)
    g, r = np.zeros(s.shape), np.zeros(s.shape)
    getattr(s, f"Compact_Filter_{DIRS[d]}_{'asym' if asym else 'sym'}")(F, g)
    o.filter(d, asym, F, r)
    assert rel_err(g, r) < TOL
    # in place (F0 aliases F), as LDDRK4 calls it
    h = F.copy()
    getattr(s, f"Compact_Filter_{DIRS[d]}_{'asym' if asym else 'sym'}")(h, h)
    assert rel_err(h, r) < TOL


@pytest.mark.parametrize("d", [0, 1, 2])
def test_gaussian_direction(pair, d):
    s, o = pair
    F = field(s, 50 + d, smooth=False)
    g, r = np.zeros(s.shape), np.zeros(s.shape)
    getattr(s, f"Gaussian_Filter_{DIRS[d]}")(F, g)
    o.gauss(d, F, r)
    assert rel_err(g, r) < TOL


def test_compact_and_gaussian_filter_multi(pair):
    s, o = pair
    F = np.ascontiguousarray(np.stack([field(s, 60 + k) for k in range(5)]))
    g, r = np.zeros_like(F), np.zeros_like(F)
    s.Compact_Filter(F, g, 5)
    o.compact_filter(F, r, 5)
    assert rel_err(g, r) < TOL
    s.Gaussian_Filter(F, g, 5)
    o.gaussian_filter(F, r, 5)
    assert rel_err(g, r) < TOL


def test_device_tensor_arguments(pair):
    """Device pointers are used in place (no host staging)."""
    import torch
    s, o = pair
    F = field(s, 70)
    r = np.zeros(s.shape)
    o.dfd(1, 0, F, r, 0, 1.0)
    Ft = torch.from_numpy(F).cuda()
    gt = torch.zeros_like(Ft)
    s.DFDY_sym(Ft, gt, 0, 1.0)
    assert rel_err(gt.cpu().numpy(), r) < TOL


@pytest.mark.parametrize("nper", [0, 1])
def test_general_tridiagonal(pair, oracle_mod, nper):
    s, _ = pair
    rng = np.random.default_rng(5)
    n, lot = 40, 300
    A = rng.uniform(0.1, 0.4, (n, lot)); C = rng.uniform(0.1, 0.4, (n, lot)); B = np.ones((n, lot))
    R = rng.normal(size=(n, lot))
    g, r = R.copy(), R.copy()
    s.tridiagonal(A, B, C, g, n, lot, nper)
    oracle_mod.tridiagonal(A, B, C, r, nper)
    assert rel_err(g, r) < TOL


@pytest.mark.parametrize("nper", [0, 1])
def test_general_pentadiagonal(pair, oracle_mod, nper):
    s, _ = pair
    rng = np.random.default_rng(6)
    n, lot = 40, 300
    A, B, D, E = (rng.uniform(0.05, 0.2, (n, lot)) for _ in range(4))
    C = np.ones((n, lot))
    R = rng.normal(size=(n, lot))
    g, r = R.copy(), R.copy()
    s.pentadiagonal(A, B, C, D, E, g, n, lot, nper)
    oracle_mod.pentadiagonal(A, B, C, D, E, r, nper)
    assert rel_err(g, r) < TOL
