"""Manufactured solutions of the Euler part of RHS, checked on the oracle.

src/mms_test_stuff.f holds the source terms the reference's authors added to
Qrhs to verify RHS against manufactured solutions (blocks dated 4/18/08,
4/20/08, 4/25/08 and the "cancelling terms" block).  Each block is the exact
flux divergence -RHS of a smooth periodic state.  Read back from the source
terms, the states are:

  A (4/18/08): rho = 1, P = 100, u = sin(x+pi/6), v = sin(y+pi/3), w = sin(z+pi/2)
  B (4/20/08): u = v = w = 1, rho = rho0 + f, P = P0 + f
  C (4/25/08): u = v = w = 1, rho = rho0 + f, P constant
  D (cancelling terms): u = v = w = 1, rho constant, P = P0 + f

with f = sin(x+pi/6) sin(y+pi/3) sin(z+pi/2).  On the periodic box
(src/rhsv_periodic_sf.f) with a negligible molecular viscosity (Re = 1e30),
RHS + source must vanish up to the sixth-order truncation error of the compact
derivatives: small on 32^3, and shrinking by about 2^6 from 16^3 to 32^3.
This pins the oracle's flux assembly to the equations themselves, not to a
restatement of the reference.

The file's last block ("viscous part only", 5/28/08) is checked through the
difference of two RHS evaluations, one with mu = 1 and one with a negligible
viscosity, which leaves the viscous terms alone."""
import math

import numpy as np
import pytest

GAMMA = 1.4
FAC2 = GAMMA / (GAMMA - 1.0)
A, B, C = math.pi / 6, math.pi / 3, math.pi / 2


def grid(n):
    """Coordinates on the (Mx, Mz, My) array: x_i = (i-1) 2 pi / n."""
    t = 2 * math.pi * np.arange(n) / n
    return t[:, None, None], t[None, None, :], t[None, :, None]   # x, y, z


def case_state_and_source(case, n):
    x, y, z = grid(n)
    shape = (n, n, n)
    sx, sy, sz = np.sin(x + A), np.sin(y + B), np.sin(z + C)
    cx, cy, cz = np.cos(x + A), np.cos(y + B), np.cos(z + C)
    src = np.zeros((5,) + shape)          # order of Q: rho u, rho v, rho w, rho, rho E
    if case == "A":
        rho = np.ones(shape)
        P = np.full(shape, 100.0)
        u, v, w = sx + 0 * y + 0 * z, sy + 0 * x + 0 * z, sz + 0 * x + 0 * y
        src[3] = cx + cy + cz
        src[0] = np.sin(2 * x + 2 * A) + sx * cy + sx * cz
        src[1] = np.sin(2 * y + 2 * B) + sy * cx + sy * cz
        src[2] = np.sin(2 * z + 2 * C) + sz * cx + sz * cy
        src[4] = (FAC2 * P * (cx + cy + cz)
                  + 1.5 * (sx * sx * cx + sy * sy * cy + sz * sz * cz)
                  + 0.5 * (sy * sy * cx + sz * sz * cx + sx * sx * cy + sz * sz * cy + sx * sx * cz + sy * sy * cz))
    else:
        f = sx * sy * sz
        df = cx * sy * sz + sx * cy * sz + sx * sy * cz      # f_x + f_y + f_z
        fx, fy, fz = cx * sy * sz, sx * cy * sz, sx * sy * cz
        u = v = w = np.ones(shape)
        if case == "B":
            rho, P = 2.0 + f, 100.0 + f
            src[3] = df
            src[0], src[1], src[2] = df + fx, df + fy, df + fz
            src[4] = (1.5 + FAC2) * df
        elif case == "C":
            rho, P = 2.0 + f, np.full(shape, 100.0)
            src[3] = df
            src[0] = src[1] = src[2] = df
            src[4] = 1.5 * df
        else:   # D
            rho, P = np.full(shape, 2.0), 100.0 + f
            src[0], src[1], src[2] = fx, fy, fz
            src[4] = FAC2 * df
    u, v, w = (np.broadcast_to(a, shape) for a in (u, v, w))
    Q = np.empty((5,) + shape)
    Q[0], Q[1], Q[2], Q[3] = rho * u, rho * v, rho * w, rho
    Q[4] = P / (GAMMA - 1.0) + 0.5 * rho * (u * u + v * v + w * w)
    return np.ascontiguousarray(Q), np.broadcast_to(src, (5,) + shape)


def residual(oracle_mod, case, n):
    from shock_turbulence_b200 import periodic_params
    p = periodic_params(n, re=1.0e30, gamma=GAMMA)
    o = oracle_mod.Oracle(p)
    Q, src = case_state_and_source(case, n)
    R = np.zeros_like(Q)
    o.rhs(Q.copy(), R, None)
    scale = max(np.abs(src).max(), 1.0)
    return [float(np.abs(R[l] + src[l]).max() / scale) for l in range(5)]


@pytest.mark.parametrize("case", ["A", "B", "C", "D"])
def test_rhs_cancels_manufactured_source(oracle_mod, case):
    e16 = residual(oracle_mod, case, 16)
    e32 = residual(oracle_mod, case, 32)
    for l in range(5):
        assert e32[l] < 1e-6, (case, l, e32[l])
        # sixth-order convergence where the error is above rounding
        if e16[l] > 1e-11:
            assert e16[l] / max(e32[l], 1e-16) > 2 ** 5.3, (case, l, e16[l], e32[l])


def test_mf_rhs_cancels_manufactured_source(oracle_mod):
    """The same check on the two-species octant family (src/rhsv_sym_mf.f),
    with Y = 1, Re = 0 (no molecular viscosity) and the state of block A
    without phase shifts: rho u = sin x is odd about x = 0 and every other
    field is even there, the parities the reference's sym/asym derivative
    choices assume at the symmetry planes.  A wrong sym/asym choice would leave
    an O(1) error at those planes.  The one-sided closures at the far faces
    are third order, so the residual over the whole octant must fall at least
    2^2.8-fold from 32^3 to 64^3 (measured: 8x in the momenta, 17x in mass and
    energy)."""
    from shock_turbulence_b200.params import default_params
    L = 2 * math.pi

    def res(n):
        p = default_params(n, length=L, gamma1=GAMMA, gamma2=GAMMA)
        o = oracle_mod.Oracle(p)
        t = np.arange(n) * (L / (n - 1))
        x, y, z = t[:, None, None], t[None, None, :], t[None, :, None]
        shape = (n, n, n)
        zero = np.zeros(shape)
        sx, sy, sz = np.sin(x) + zero, np.sin(y) + zero, np.sin(z) + zero
        cx, cy, cz = np.cos(x) + zero, np.cos(y) + zero, np.cos(z) + zero
        P = 100.0
        Q = np.empty((5,) + shape)
        Q[0], Q[1], Q[2], Q[3] = sx, sy, sz, 1.0
        Q[4] = P / (GAMMA - 1.0) + 0.5 * (sx * sx + sy * sy + sz * sz)
        src = np.empty_like(Q)
        src[3] = cx + cy + cz
        src[0] = np.sin(2 * x) + sx * cy + sx * cz
        src[1] = np.sin(2 * y) + sy * cx + sy * cz
        src[2] = np.sin(2 * z) + sz * cx + sz * cy
        src[4] = (FAC2 * P * (cx + cy + cz) + 1.5 * (sx * sx * cx + sy * sy * cy + sz * sz * cz)
                  + 0.5 * (sy * sy * cx + sz * sz * cx + sx * sx * cy + sz * sz * cy + sx * sx * cz + sy * sy * cz))
        Y = np.ones(shape)
        o.set_state(Q, Y)
        o.compute_gamma(Y)
        R = np.zeros_like(Q)
        o.rhs(Q.copy(), R, Y)
        scale = np.abs(src).max()
        return [float(np.abs(R[l] + src[l]).max() / scale) for l in range(5)]

    e32, e64 = res(32), res(64)
    for l in range(5):
        assert e64[l] < 2e-5, (l, e64[l])
        assert e32[l] / e64[l] > 2 ** 2.8, (l, e32[l], e64[l])


def viscous_state(n, h):
    """The block "MMS source terms for viscous part only" (5/28/08): rho = 1,
    P = 100 and u = (sin x cos y cos z, cos x sin y cos z, cos x cos y sin z).
    With mu = 1 the viscous terms of RHS equal -source: -4 u_i in the momenta
    and -4|u|^2 + 4 (s_xy^2 + s_xz^2 + s_yz^2) in the energy (u_i d_j tau_ij
    plus the dissipation tau_ij d_j u_i, the diagonal of tau being zero)."""
    t = np.arange(n) * h
    x, y, z = t[:, None, None], t[None, None, :], t[None, :, None]
    zero = np.zeros((n, n, n))
    a = np.sin(x) * np.cos(y) * np.cos(z) + zero
    b = np.cos(x) * np.sin(y) * np.cos(z) + zero
    c = np.cos(x) * np.cos(y) * np.sin(z) + zero
    sxy = np.sin(x) * np.sin(y) * np.cos(z) + zero
    sxz = np.sin(x) * np.cos(y) * np.sin(z) + zero
    syz = np.cos(x) * np.sin(y) * np.sin(z) + zero
    P = 100.0
    Q = np.empty((5, n, n, n))
    Q[0], Q[1], Q[2], Q[3] = a, b, c, 1.0
    Q[4] = P / (GAMMA - 1.0) + 0.5 * (a * a + b * b + c * c)
    src = np.zeros_like(Q)
    src[0], src[1], src[2] = 4 * a, 4 * b, 4 * c
    src[4] = 4 * (a * a + b * b + c * c) - 4 * (sxy ** 2 + sxz ** 2 + syz ** 2)
    return Q, src


def viscous_residual(oracle_mod, make_params, n, h, with_y):
    """RHS with mu = 1 (Re = 1, vis_exp = 0) minus RHS with a negligible
    viscosity (Re = 1e30) is the viscous part alone; its residual against the
    source, relative to max|source|, per conserved field."""
    Q, src = viscous_state(n, h)
    Y = np.ones(Q.shape[1:]) if with_y else None
    out = []
    for re in (1.0, 1.0e30):
        o = oracle_mod.Oracle(make_params(re))
        if with_y:
            o.set_state(Q, Y)
            o.compute_gamma(Y)
        R = np.zeros_like(Q)
        o.rhs(Q.copy(), R, Y)
        out.append(R)
    V = out[0] - out[1]
    scale = np.abs(src).max()
    return [float(np.abs(V[l] + src[l]).max() / scale) for l in range(5)]


def test_periodic_viscous_part_cancels_manufactured_source(oracle_mod):
    """Periodic box (src/rhsv_periodic_sf.f, mu = ((gamma-1)T)^vis_exp / Re):
    sixth-order convergence, measured 1.5e-6 on 16^3 and 2.4e-8 on 32^3."""
    from shock_turbulence_b200 import periodic_params

    def res(n):
        return viscous_residual(oracle_mod, lambda re: periodic_params(n, re=re, gamma=GAMMA, vis_exp=0.0),
                                n, 2 * math.pi / n, False)

    e16, e32 = res(16), res(32)
    assert e16[3] == 0.0 and e32[3] == 0.0        # no viscous term in the mass equation
    for l in (0, 1, 2, 4):
        assert e32[l] < 1e-7, (l, e32[l])
        assert e16[l] / e32[l] > 2 ** 5.3, (l, e16[l], e32[l])


def test_mf_viscous_part_cancels_manufactured_source(oracle_mod):
    """_mf octant (src/rhsv_sym_mf.f) with Y = 1 and Re = Re1 = 1 (the viscous
    term is added because Re > 0): u is odd about its own symmetry plane and
    even about the others, as the sym/asym closures assume.  The far faces'
    one-sided second-derivative closures set the rate: measured 6.7e-3 on
    32^3 and 8.6e-4 on 64^3 in the momenta, 4.5e-3 and 2.7e-4 in the energy."""
    from shock_turbulence_b200.params import default_params
    L = 2 * math.pi

    def res(n):
        return viscous_residual(
            oracle_mod, lambda re: default_params(n, length=L, gamma1=GAMMA, gamma2=GAMMA, re=re, re1=re,
                                                  vis_exp=0.0),
            n, L / (n - 1), True)

    e32, e64 = res(32), res(64)
    assert e32[3] == 0.0 and e64[3] == 0.0
    for l in (0, 1, 2, 4):
        assert e64[l] < 2e-3, (l, e64[l])
        assert e32[l] / e64[l] > 2 ** 2.5, (l, e32[l], e64[l])
