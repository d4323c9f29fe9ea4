"""Output-side diagnostics of the oracle (Compute_Grad src/grad_sym.f:13-120,
Compute_SRM_Stats pproc/pproc_mf.f:4-186, Generate_Shock_Surface
src/shock.f:163-260): analytic cases, and a loop-for-loop numpy restatement
of the shell statistics and the shock surface on random fields."""
import numpy as np
import pytest

from shock_turbulence_b200.params import default_params

N = 32


@pytest.fixture(scope="module")
def orc(oracle_mod):
    return oracle_mod.Oracle(default_params(N))


def coords(p):
    x = p.x_start + p.x_leng * np.arange(p.nx) / (p.nx - 1)
    y = p.y_start + p.y_leng * np.arange(p.ny) / (p.ny - 1)
    z = p.z_start + p.z_leng * np.arange(p.nz) / (p.nz - 1)
    return x, y, z


def state_from_velocity(o, u, v, w, Y=None):
    Q = np.empty((5,) + o.shape)
    Q[0], Q[1], Q[2], Q[3], Q[4] = u, v, w, 1.0, 2.5
    Y = np.full(o.shape, 0.5) if Y is None else Y
    o.set_state(Q, Y)
    return Q, Y


def test_fluid_at_rest(orc):
    z = np.zeros(orc.shape)
    state_from_velocity(orc, z, z, z)
    G, maxdil, ens = orc.compute_grad()
    assert np.abs(G).max() == 0.0 and maxdil == 0.0 and ens == 0.0


def test_linear_expansion(orc):
    """u = a (x, y, z): dilatation 3a, no vorticity (the compact schemes are
    exact on linear fields, the odd reflection included)."""
    p = orc.params
    x, y, z = coords(p)
    a = 0.7
    X = np.broadcast_to(x[:, None, None], orc.shape)
    Yc = np.broadcast_to(y[None, None, :], orc.shape)
    Z = np.broadcast_to(z[None, :, None], orc.shape)
    state_from_velocity(orc, a * X, a * Yc, a * Z)
    G, maxdil, ens = orc.compute_grad()
    assert np.allclose(G[3], 3 * a, rtol=1e-10, atol=0)
    assert np.abs(G[:3]).max() < 1e-9
    assert abs(maxdil - 3 * a) < 1e-10 and ens < 1e-16


def test_constant_mass_fraction_mixing_width(orc):
    c = 0.3
    state_from_velocity(orc, np.zeros(orc.shape), np.zeros(orc.shape), np.zeros(orc.shape), np.full(orc.shape, c))
    hmix, tke, ur, ya = orc.compute_srm_stats()
    full = np.isfinite(ya)
    assert np.allclose(ya[full], c, rtol=1e-14)
    dx = orc.params.x_leng / (N - 1)
    assert hmix == pytest.approx(full.sum() * 8 * c * (1 - c) * dx * np.sqrt(3.0), rel=1e-13)
    assert tke == 0.0 and np.all(ur[full] == 0.0)


def shell_stats_numpy(p, Q, Y):
    """pproc/pproc_mf.f:4-186 and src/auxiliary_mf.f:266-332 restated with
    numpy (bins by comparison, sums per bin)."""
    x, y, z = coords(p)
    dx = x[1] - x[0]
    dy = y[1] - y[0]
    dz = z[1] - z[0]
    na = p.nx // 2 + 10 * (p.nx // 128)
    I = np.arange(p.nx)[:, None, None].astype(float)
    J = np.arange(p.ny)[None, None, :].astype(float)
    K = np.arange(p.nz)[None, :, None].astype(float)
    rad = np.sqrt((I * dx) ** 2 + (J * dy) ** 2 + (K * dz) ** 2) * np.ones(Y.shape)
    U = Q[:3] / Q[3]
    with np.errstate(invalid="ignore", divide="ignore"):
        Ur = (x[:, None, None] / rad) * U[0] + (y[None, None, :] / rad) * U[1] + (z[None, :, None] / rad) * U[2]
    Ur[0, 0, 0] = 0.0
    rs = np.zeros(na + 1)
    for M in range(2, na + 2):
        rs[M - 1] = rs[M - 2] + (dx * 2.0 * np.sqrt(3.0) if M <= 4 else dx * np.sqrt(3.0))
    ru = np.concatenate([[0.0], np.cumsum(np.full(na, dx * np.sqrt(3.0)))])

    def avg(F, r):
        out = np.zeros(na)
        for M in range(na):
            sel = (rad >= r[M]) & (rad < r[M + 1])
            with np.errstate(invalid="ignore"):
                out[M] = F[sel].sum() / sel.sum()
        return out
    ura, ya = avg(Ur, rs), avg(Y, rs)
    tke = np.zeros(Y.shape)
    inner = (I > 0) & (J > 0) & (K > 0)
    for M in range(na):
        sel = (rad >= ru[M]) & (rad < ru[M + 1])
        urp2 = (Ur - ura[M]) ** 2
        with np.errstate(invalid="ignore", divide="ignore"):
            t1 = np.where(inner, U[0] - Ur * (I * dx / rad), 0.0)
            t2 = np.where(inner, U[1] - Ur * (J * dy / rad), 0.0)
            t3 = np.where(inner, U[2] - Ur * (K * dz / rad), 0.0)
        tke[sel] = (t1 ** 2 + t2 ** 2 + t3 ** 2 + urp2)[sel]
    tke_total = tke.sum() / Y.size
    sel = (ya > 0) & (ya < 1)
    hmix = (8 * ya[sel] * (1 - ya[sel]) * dx * np.sqrt(3.0)).sum()
    return hmix, tke_total, ura, ya


def test_shell_statistics_against_numpy(orc):
    rng = np.random.default_rng(4)
    u, v, w = (0.1 * rng.standard_normal(orc.shape) for _ in range(3))
    Y = rng.uniform(0.0, 1.0, orc.shape)
    Q, Y = state_from_velocity(orc, u, v, w, Y)
    hmix, tke, ur, ya = orc.compute_srm_stats()
    h2, t2, ur2, ya2 = shell_stats_numpy(orc.params, Q, Y)
    assert hmix == pytest.approx(h2, rel=1e-12)
    assert tke == pytest.approx(t2, rel=1e-12)
    assert np.allclose(ur, ur2, rtol=1e-11, atol=1e-15, equal_nan=True)
    assert np.allclose(ya, ya2, rtol=1e-12, equal_nan=True)


def test_shock_surface_against_numpy(orc):
    rng = np.random.default_rng(5)
    beta = rng.uniform(0.0, 1.0, orc.shape) ** 4
    orc.set_state(np.ones((5,) + orc.shape), np.ones(orc.shape))
    orc.set_common("beta_hyper", beta)
    ra, sk = orc.shock_surface()
    x, y, z = coords(orc.params)
    sel = beta > 0.1 * beta.max()
    X = np.broadcast_to(x[:, None, None], orc.shape)[sel]
    Yc = np.broadcast_to(y[None, None, :], orc.shape)[sel]
    Z = np.broadcast_to(z[None, :, None], orc.shape)[sel]
    n = sel.sum()
    r = np.sqrt((X - X.sum() / n) ** 2 + (Yc - Yc.sum() / n) ** 2 + (Z - Z.sum() / n) ** 2)
    ra2 = r.sum() / n
    sk2 = np.sqrt(((r - ra2) ** 2).sum()) / (n * ra2)
    assert ra == pytest.approx(ra2, rel=1e-12) and sk == pytest.approx(sk2, rel=1e-12)
