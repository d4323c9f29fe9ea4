"""Line solves whose segment count is odd or below 32, against the oracle.

A line of n points is cut into P = n/S segments (S the smallest of 2, 3, 4,
6, 8, 12, 16 with n/S <= 32) and a CTA runs 16 lines x P segments, 16 P
threads.  The compact filter scans its segment carries across the CTA; the
tridiagonal solves of short segments scan theirs one line per warp.  With P
odd (n = 272: S = 16, P = 17) the CTA ends in a half warp, which takes no
line; with P < 32 the warps take more than one line each (n = 48: P = 24,
12 warps for 16 lines; n = 80: P = 20).  Both families (_mf symmetric octant
and periodic), every operator and direction, a whole _mf step, and the FP32
mode's step against the FP64 one (on 272 x 160 x 80: the FP32 mode needs
ny to be a multiple of 32)."""
import numpy as np
import pytest

from conftest import rel_err
from shock_turbulence_b200.params import PRECISION_FP32, default_params, periodic_params

pytestmark = pytest.mark.gpu
GRID = (272, 48, 80)
DIRS = "XYZ"


def mf_params(**kw):
    return default_params(*GRID, length=2.0, re=100.0, c_beta_scale=1.75, **kw)


def field(shape, seed):
    return np.random.default_rng(seed).standard_normal(shape)


@pytest.fixture(scope="module")
def mf_pair(oracle_mod):
    from shock_turbulence_b200 import Solver
    p = mf_params()
    s = Solver(p)
    yield s, oracle_mod.Oracle(p)
    s.close()


@pytest.fixture(scope="module")
def per_pair(oracle_mod):
    from shock_turbulence_b200 import Solver
    p = periodic_params(272, 48, 16)
    s = Solver(p)
    yield s, oracle_mod.Oracle(p)
    s.close()


@pytest.mark.parametrize("d", [0, 1, 2])
@pytest.mark.parametrize("asym", [0, 1])
def test_mf_operators(mf_pair, d, asym):
    s, o = mf_pair
    sfx = "_asym" if asym else "_sym"
    F = field(s.shape, 10 + d + 3 * asym)
    g, r = field(s.shape, 20 + d), None
    r = g.copy()
    getattr(s, f"DFD{DIRS[d]}{sfx}")(F, g, 1, -0.5)
    o.dfd(d, asym, F, r, 1, -0.5)
    assert rel_err(g, r) < 1e-12, "DFD"
    g1, g2, r1, r2 = (np.zeros(s.shape) for _ in range(4))
    getattr(s, f"D2FD{DIRS[d]}2{sfx}")(F, g1, g2, 1)
    o.d2fd2(d, asym, F, r1, r2, 1)
    assert rel_err(g2, r2) < 1e-12 and rel_err(g1, r1) < 1e-12, "D2FD2"
    g, r = np.zeros(s.shape), np.zeros(s.shape)
    getattr(s, f"Compact_Filter_{DIRS[d]}{sfx}")(F, g)
    o.filter(d, asym, F, r)
    assert rel_err(g, r) < 1e-12, "filter"


@pytest.mark.parametrize("d", [0, 1, 2])
def test_periodic_operators(per_pair, d):
    s, o = per_pair
    F = field(s.shape, 30 + d)
    g = field(s.shape, 40 + d)
    r = g.copy()
    getattr(s, "DFD" + DIRS[d])(F, g, 1, -0.5)
    o.dfd(d, 0, F, r, 1, -0.5)
    assert rel_err(g, r) < 1e-12, "DFD"
    g1, g2, r1, r2 = (np.zeros(s.shape) for _ in range(4))
    getattr(s, "D2FD" + DIRS[d] + "2")(F, g1, g2, 1)
    o.d2fd2(d, 0, F, r1, r2, 1)
    assert rel_err(g2, r2) < 1e-12 and rel_err(g1, r1) < 1e-12, "D2FD2"
    g, r = np.zeros(s.shape), np.zeros(s.shape)
    getattr(s, "Compact_Filter_" + DIRS[d])(F, g)
    o.filter(d, 0, F, r)
    assert rel_err(g, r) < 1e-12, "filter"


def blast(p, seed=7):
    from shock_turbulence_b200.initial import blast_in_turbulence
    return blast_in_turbulence(p, k0=4, mach_t=0.1, p_ratio=20.0, radius_cells=4, seed=seed)


def test_mf_step(mf_pair):
    s, o = mf_pair
    Q, Y = blast(s.params)
    for h in (s, o):
        h.set_state(Q, Y)
    s.Compute_gamma(Y); o.compute_gamma(Y)
    s.Compute_hyper(Q, Y); o.compute_hyper(Q, Y)
    ts, ks = s.step(0.0, 0)
    to, ko = o.step(0.0, 0)
    assert ks == ko == 1 and abs(ts - to) <= 1e-12 * to
    Qg, Yg = s.get_state()
    Qo, Yo = o.get_state()
    for l in range(5):
        assert rel_err(Qg[l], Qo[l]) < 1e-10, l
    assert rel_err(Yg, Yo) < 1e-10


def test_fp32_step_near_fp64():
    """The FP32 mode's line kernels (two lines per thread, 32 lines per CTA:
    ny a multiple of 32) on odd and short segmentations (x: P = 17, y: n =
    160, P = 20, z: P = 20): one step within float rounding of the FP64
    step."""
    from shock_turbulence_b200 import Solver
    out = []
    for prec in (0, PRECISION_FP32):
        p = default_params(272, 160, 80, length=2.0, re=100.0, c_beta_scale=1.75, precision=prec)
        Q, Y = blast(p)
        s = Solver(p)
        try:
            s.set_state(Q, Y)
            s.Compute_gamma(Y)
            s.Compute_hyper(Q, Y)
            s.step(0.0, 0)
            out.append(s.get_state())
        finally:
            s.close()
    (Q64, Y64), (Q32, Y32) = out
    for l in range(5):
        assert rel_err(Q32[l], Q64[l]) < 1e-5, l
    assert rel_err(Y32, Y64) < 1e-5
