"""Known answers for the oracle's boundary routines of the _mf octant.

bc_RHS (src/bc_mf.f:11-463): on a state with uniform velocity (U0, 0, 0),
rho = 1 and a pressure linear in x, the compact derivative of P is exact at
the far x face, so
the outgoing characteristic at the far x face is L5 = (u + c) dP/dx and every
other L is zero.  The LODI relations (Poinsot & Lele, J. Comput. Phys. 101,
1992) then give d(rho)/dt = -L5/(2c^2), dP/dt = -L5/2 and du/dt = -L5/(2 rho c),
which the test converts to the conserved variables itself.  On the far y and z
faces dP/dn = du_n/dn = 0, so their rows are zero (to rounding).  They are written after
the x face and overwrite its edges.  No other cell of Qrhs changes, and the
normal momentum is zeroed on the x = 0 symmetry plane of Q itself.

Sponge_Forcing (src/sponge_mf.f:7-127): Qrhs -= (sx + sy + sz)(Q - Qref) in
the outer ceil(0.1 N) points, with sigma = 4 r^3.  The ratio r is a default-REAL
(float32) quotient, src/sponge_mf.f:85-103.  Qref is the state behind a
Mach-1.8 normal shock (Rankine-Hugoniot) at rest, with base pressure 0.71429."""
import math

import numpy as np

from shock_turbulence_b200.params import default_params

G = 1.4


def test_bc_rhs_outgoing_acoustic_wave(oracle_mod):
    # The symmetric closure forces dP/dx = 0 at x = 0, an error that decays by
    # (3 - sqrt 5)/2 = 0.38 per point; 48 points bring it below 1e-19 at the
    # far face, so dP/dx is exact there to rounding.
    n, L = 48, 2.0
    o = oracle_mod.Oracle(default_params(n, length=L, gamma1=G, gamma2=G))
    x = (np.arange(n) * L / (n - 1))[:, None, None]
    U0, P0, k = 0.3, 1.0, 0.2
    P = P0 + k * x + np.zeros((n, n, n))
    Q = np.zeros((5, n, n, n))
    Q[0], Q[3] = U0, 1.0
    Q[4] = P / (G - 1.0) + 0.5 * U0 * U0
    Y = np.ones((n, n, n))
    o.set_state(Q, Y)
    o.compute_gamma(Y)
    for name in ("dux_dx", "duy_dy", "duz_dz"):
        o.set_common(name, np.zeros((n, n, n)))
    R = np.full_like(Q, 7.0)
    Yr = np.full((n, n, n), 7.0)
    Qb = Q.copy()
    o.bc_rhs(Qb, R, Y, Yr, 0.0)

    # Q: rho u zeroed on the x = 0 plane, nothing else touched
    assert np.all(Qb[0][0] == 0.0)
    Qb[0][0] = Q[0][0]
    assert np.array_equal(Qb, Q)

    # far x face (index i = n-1 of the (Mx, Mz, My) array), away from the y and z faces
    Pf = P0 + k * L
    c = math.sqrt(G * Pf)
    L5 = (U0 + c) * k
    drho, dP, du = -L5 / (2 * c * c), -L5 / 2, -L5 / (2 * c)
    expect = [U0 * drho + du,                    # d(rho u)/dt
              0.0, 0.0,
              drho,                              # d(rho)/dt
              0.5 * U0 * U0 * drho + U0 * du + dP / (G - 1.0)]   # d(rho E)/dt
    for l in range(5):
        face = R[l][n - 1, : n - 1, : n - 1]
        assert np.allclose(face, expect[l], rtol=1e-12, atol=1e-14), (l, face[0, 0], expect[l])
    assert np.all(Yr[n - 1, : n - 1, : n - 1] == 0.0)

    # far y face (last axis) and far z face (middle axis): zero rows, edges
    # included.  The one-sided closure weights are not exact binary fractions,
    # so the derivative of a constant is zero only to rounding (~1e-14 here).
    for l in range(5):
        assert np.abs(R[l][:, :, n - 1]).max() < 1e-12, l
        assert np.abs(R[l][:, n - 1, :]).max() < 1e-12, l
    assert np.all(Yr[:, :, n - 1] == 0.0) and np.all(Yr[:, n - 1, :] == 0.0)

    # every other cell untouched
    assert np.all(R[:, : n - 1, : n - 1, : n - 1] == 7.0)
    assert np.all(Yr[: n - 1, : n - 1, : n - 1] == 7.0)


def test_sponge_forcing_profile_and_reference_state(oracle_mod):
    n = 48                                   # ceil(4.8) = 5 sponge points: r = m/5 rounds in float32
    o = oracle_mod.Oracle(default_params(n, gamma1=G, gamma2=G))
    vals = [0.2, -0.1, 0.05, 2.0, 5.0]
    Q = np.empty((5, n, n, n))
    for l, v in enumerate(vals):
        Q[l] = v
    Y = np.full((n, n, n), 0.25)
    R = np.zeros_like(Q)
    Yr = np.zeros((n, n, n))
    o.sponge_forcing(Q, R, Y, Yr)

    Ms, pb = 1.8, 0.71429
    rho_ref = (G + 1) * Ms ** 2 / ((G - 1) * Ms ** 2 + 2)             # normal-shock density ratio
    P_ref = pb * (1 + 2 * G / (G + 1) * (Ms ** 2 - 1))                # normal-shock pressure ratio
    Qref = [0.0, 0.0, 0.0, rho_ref, P_ref / (G - 1)]

    nsp = math.ceil(0.1 * n)
    start = n - nsp
    sig = np.zeros(n)
    for q in range(n):
        gI = q + 1
        if gI >= start:
            r = np.float32(gI - start) / np.float32(nsp)             # default-REAL quotient
            sig[q] = 4.0 * float(r) ** 3
    assert float(np.float32(1) / np.float32(5)) != 0.2               # the float32 rounding is exercised
    s = sig[:, None, None] + sig[None, None, :] + sig[None, :, None]  # x, y, z on (Mx, Mz, My)
    for l in range(5):
        assert np.allclose(R[l], -s * (vals[l] - Qref[l]), rtol=1e-14, atol=0), l
    assert np.allclose(Yr, -s * (vals[3] * 0.25 - vals[3] * 1.0), rtol=1e-14, atol=0)
    # only the sponge shell is forced
    assert np.all(R[:, : start - 1, : start - 1, : start - 1] == 0.0)
    assert np.any(R[:, start:, :, :] != 0.0)
