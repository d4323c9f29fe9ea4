"""The GPU RHS against the reference's manufactured solutions
(src/mms_test_stuff.f), through the C ABI: the same states, source terms and
bounds as the oracle's check in test_oracle_mms.py, with the CUDA library
computing RHS.

- periodic box (four Euler solutions): residual below 1e-6 of the source on
  32^3, falling at least 2^5.3-fold from 16^3;
- _mf octant (Y = 1, Re = 0): residual below 2e-5 on 64^3, falling at least
  2^2.8-fold from 32^3;
- the viscous-only solution, as RHS(mu = 1) - RHS(mu ~ 0): below 1e-7 on the
  32^3 box at sixth order, below 2e-3 on the 64^3 octant at 2^2.5 per
  doubling."""
import math

import numpy as np
import pytest

from test_oracle_mms import FAC2, GAMMA, case_state_and_source

pytestmark = pytest.mark.gpu


def periodic_residual(case, n):
    from shock_turbulence_b200 import Solver, periodic_params
    s = Solver(periodic_params(n, re=1.0e30, gamma=GAMMA))
    Q, src = case_state_and_source(case, n)
    R = np.zeros_like(Q)
    s.RHS(Q.copy(), R, None)
    s.close()
    scale = max(np.abs(src).max(), 1.0)
    return [float(np.abs(R[l] + src[l]).max() / scale) for l in range(5)]


@pytest.mark.parametrize("case", ["A", "B", "C", "D"])
def test_periodic_rhs_cancels_manufactured_source(case):
    e16 = periodic_residual(case, 16)
    e32 = periodic_residual(case, 32)
    for l in range(5):
        assert e32[l] < 1e-6, (case, l, e32[l])
        if e16[l] > 1e-11:
            assert e16[l] / max(e32[l], 1e-16) > 2 ** 5.3, (case, l, e16[l], e32[l])


def mf_residual(n):
    from shock_turbulence_b200 import Solver
    from shock_turbulence_b200.params import default_params
    L = 2 * math.pi
    s = Solver(default_params(n, length=L, gamma1=GAMMA, gamma2=GAMMA))
    t = np.arange(n) * (L / (n - 1))
    x, y, z = t[:, None, None], t[None, None, :], t[None, :, None]
    zero = np.zeros((n, n, n))
    sx, sy, sz = np.sin(x) + zero, np.sin(y) + zero, np.sin(z) + zero
    cx, cy, cz = np.cos(x) + zero, np.cos(y) + zero, np.cos(z) + zero
    P = 100.0
    Q = np.empty((5, n, n, n))
    Q[0], Q[1], Q[2], Q[3] = sx, sy, sz, 1.0
    Q[4] = P / (GAMMA - 1.0) + 0.5 * (sx * sx + sy * sy + sz * sz)
    src = np.empty_like(Q)
    src[3] = cx + cy + cz
    src[0] = np.sin(2 * x) + sx * cy + sx * cz
    src[1] = np.sin(2 * y) + sy * cx + sy * cz
    src[2] = np.sin(2 * z) + sz * cx + sz * cy
    src[4] = (FAC2 * P * (cx + cy + cz) + 1.5 * (sx * sx * cx + sy * sy * cy + sz * sz * cz)
              + 0.5 * (sy * sy * cx + sz * sz * cx + sx * sx * cy + sz * sz * cy + sx * sx * cz + sy * sy * cz))
    Y = np.ones((n, n, n))
    s.set_state(Q, Y)
    s.Compute_gamma(Y)
    R = np.zeros_like(Q)
    s.RHS(Q.copy(), R, Y)
    s.close()
    scale = np.abs(src).max()
    return [float(np.abs(R[l] + src[l]).max() / scale) for l in range(5)]


def test_mf_rhs_cancels_manufactured_source():
    e32, e64 = mf_residual(32), mf_residual(64)
    for l in range(5):
        assert e64[l] < 2e-5, (l, e64[l])
        assert e32[l] / e64[l] > 2 ** 2.8, (l, e32[l], e64[l])


def gpu_viscous_residual(make_params, n, h, with_y):
    """The CUDA RHS with mu = 1 minus the CUDA RHS with a negligible viscosity,
    against the viscous-only source of src/mms_test_stuff.f."""
    from shock_turbulence_b200 import Solver
    from test_oracle_mms import viscous_state
    Q, src = viscous_state(n, h)
    Y = np.ones(Q.shape[1:]) if with_y else None
    out = []
    for re in (1.0, 1.0e30):
        s = Solver(make_params(re))
        if with_y:
            s.set_state(Q, Y)
            s.Compute_gamma(Y)
        R = np.zeros_like(Q)
        s.RHS(Q.copy(), R, Y)
        s.close()
        out.append(R)
    V = out[0] - out[1]
    scale = np.abs(src).max()
    return [float(np.abs(V[l] + src[l]).max() / scale) for l in range(5)]


def test_periodic_viscous_part_cancels_manufactured_source():
    from shock_turbulence_b200 import periodic_params
    e16, e32 = (gpu_viscous_residual(lambda re: periodic_params(n, re=re, gamma=GAMMA, vis_exp=0.0),
                                     n, 2 * math.pi / n, False) for n in (16, 32))
    for l in (0, 1, 2, 4):
        assert e32[l] < 1e-7, (l, e32[l])
        assert e16[l] / e32[l] > 2 ** 5.3, (l, e16[l], e32[l])


def test_mf_viscous_part_cancels_manufactured_source():
    from shock_turbulence_b200.params import default_params
    L = 2 * math.pi
    e32, e64 = (gpu_viscous_residual(
        lambda re: default_params(n, length=L, gamma1=GAMMA, gamma2=GAMMA, re=re, re1=re, vis_exp=0.0),
        n, L / (n - 1), True) for n in (32, 64))
    for l in (0, 1, 2, 4):
        assert e64[l] < 2e-3, (l, e64[l])
        assert e32[l] / e64[l] > 2 ** 2.5, (l, e32[l], e64[l])
