"""Periodic single-fluid family on the GPU against the oracle
(src/derivCDopt6_periodic.f, src/filters_periodic.f, src/rhsv_periodic_sf.f,
src/hyper_dynamic.f, src/hyper_rhs.f, src/lddrk4_periodic_sf.f).

Tolerances as for the _mf family: 1e-12 per line operator, 1e-11 for the RHS,
1e-10 for the artificial-viscosity fields and after full LDDRK4 steps."""
import ctypes

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

GRID = (32, 48, 16)
TOL = 1e-12
ST_E_UNSUPPORTED = -4


def params(grid=GRID, **kw):
    from shock_turbulence_b200 import periodic_params
    return periodic_params(*grid, **kw)


def state(p, seed=3, urms=0.1):
    from shock_turbulence_b200.initial import periodic_turbulence
    return periodic_turbulence(p, k0=4.0, urms=urms, seed=seed)


@pytest.fixture(scope="module")
def pair(oracle_mod):
    from shock_turbulence_b200 import Solver
    p = params()
    return Solver(p), oracle_mod.Oracle(p)


def field(s, seed):
    return np.random.default_rng(seed).standard_normal(s.shape)


@pytest.mark.parametrize("d", [0, 1, 2])
@pytest.mark.parametrize("iadd", [0, 1])
def test_first_derivative(pair, d, iadd):
    s, o = pair
    F = field(s, 10 + d)
    g, r = field(s, 20 + d), None
    r = g.copy()
    getattr(s, "DFD" + "XYZ"[d])(F, g, iadd, -0.5)
    o.dfd(d, 0, F, r, iadd, -0.5)
    assert rel_err(g, r) < TOL


@pytest.mark.parametrize("d", [0, 1, 2])
@pytest.mark.parametrize("iadd", [0, 1])
def test_second_derivative(pair, d, iadd):
    s, o = pair
    F = field(s, 30 + d)
    g1, g2, r1, r2 = (np.zeros(s.shape) for _ in range(4))
    getattr(s, "D2FD" + "XYZ"[d] + "2")(F, g1 if iadd else None, g2, iadd)
    o.d2fd2(d, 0, F, r1, r2, iadd)
    assert rel_err(g2, r2) < TOL
    if iadd:
        assert rel_err(g1, r1) < TOL


@pytest.mark.parametrize("d", [0, 1, 2])
def test_filters(pair, d):
    s, o = pair
    F = field(s, 40 + d)
    g, r = np.zeros(s.shape), np.zeros(s.shape)
    getattr(s, "Compact_Filter_" + "XYZ"[d])(F, g)
    o.filter(d, 0, F, r)
    assert rel_err(g, r) < TOL
    g, r = np.zeros(s.shape), np.zeros(s.shape)
    getattr(s, "Gaussian_Filter_" + "XYZ"[d])(F, g)
    o.gauss(d, F, r)
    assert rel_err(g, r) < TOL
    # in place, as Compact_Filter calls it (src/filters_periodic.f:104-106)
    g = F.copy()
    getattr(s, "Compact_Filter_" + "XYZ"[d])(g, g)
    o.filter(d, 0, F, r)
    assert rel_err(g, r) < TOL


def test_multi_field_filters(pair):
    s, o = pair
    F = np.random.default_rng(50).standard_normal((5,) + s.shape)
    g, r = np.zeros_like(F), np.zeros_like(F)
    s.Compact_Filter(F, g, 5)
    o.compact_filter(F, r, 5)
    assert rel_err(g, r) < TOL
    g, r = np.zeros_like(F), np.zeros_like(F)
    s.Gaussian_Filter(F, g, 5)
    o.gaussian_filter(F, r, 5)
    assert rel_err(g, r) < TOL


def test_rhs_and_artificial_viscosity(pair):
    s, o = pair
    Q = state(s.params)
    Qg, Qo = Q.copy(), Q.copy()
    Rg, Ro = np.zeros_like(Q), np.zeros_like(Q)
    s.RHS(Qg, Rg)
    o.rhs(Qo, Ro)
    for f in range(5):
        assert rel_err(Rg[f], Ro[f]) < 1e-11, f
    assert rel_err(Qg, Qo) < 1e-14        # the momentum round trip of RHS_yz
    s.Compute_hyper(Qg)
    o.compute_hyper(Qo)
    for name in ("beta_hyper", "visc_hyper", "k_hyper"):
        assert rel_err(s.get_common(name), o.get_common(name)) < 1e-10, name
    s.Hyper_RHS(Qg, Rg)
    o.hyper_rhs(Qo, Ro)
    for f in range(5):
        assert rel_err(Rg[f], Ro[f]) < 1e-10, f


def test_fix_pressure_base_value(pair):
    s, o = pair
    Q = state(s.params)
    Q[4, 0, 0, :4] = 0.0                 # negative pressure in a few cells
    g, r = Q.copy(), Q.copy()
    s.Fix_Pressure(g)
    o.fix_pressure(r)
    assert rel_err(g, r) < 1e-15
    P = (1.4 - 1.0) * (g[4] - 0.5 * (g[0] ** 2 + g[1] ** 2 + g[2] ** 2) / g[3])
    assert np.allclose(P[0, 0, :4], 0.71463, rtol=1e-12)


@pytest.mark.parametrize("rk_mode", [0, 1])
def test_lddrk4_steps(oracle_mod, rk_mode):
    from shock_turbulence_b200 import Solver
    p = params(rk_mode=rk_mode)
    s, o = Solver(p), oracle_mod.Oracle(p)
    Q = state(p, seed=5, urms=0.15)
    s.set_state(Q)
    o.set_state(Q, None)
    s.Compute_hyper(Q)
    o.compute_hyper(Q)
    tg = to = 0.0
    sg = so = 0
    for _ in range(3):
        tg, sg = s.step(tg, sg)
        to, so = o.step(to, so)
    Qg, _ = s.get_state()
    Qo, _ = o.get_state()
    for f in range(5):
        assert rel_err(Qg[f], Qo[f]) < 1e-10, f
    assert abs(tg - to) < 1e-12 * to and sg == so == 3
    mg, mo = s.monitors(), o.monitors()
    for k in (0, 4, 5, 6):
        assert abs(mg[k] - mo[k]) <= 1e-11 * abs(mo[k]), k


def test_config0_ten_steps_match_and_conserve_mass(oracle_mod):
    """The 64^3 periodic decaying-turbulence case (Re 100, Pr 0.7, artificial
    viscosity on, CFL 0.5, 10 LDDRK4 steps)."""
    from shock_turbulence_b200 import Solver
    p = params((64, 64, 64), re=100.0, pr=0.7, cfl_cal=0.5)
    s, o = Solver(p), oracle_mod.Oracle(p)
    Q = state(p, seed=0)
    s.set_state(Q)
    o.set_state(Q, None)
    s.Compute_hyper(Q)
    o.compute_hyper(Q)
    tg = to = 0.0
    sg = so = 0
    for _ in range(10):
        tg, sg = s.step(tg, sg)
        to, so = o.step(to, so)
    Qg, _ = s.get_state()
    Qo, _ = o.get_state()
    for f in range(5):
        assert rel_err(Qg[f], Qo[f]) < 1e-10, f
    assert abs(Qg[3].mean() - Q[3].mean()) < 1e-13


def test_family_routines_are_separate(pair):
    from shock_turbulence_b200 import Solver, default_params
    s, _ = pair
    F = field(s, 60)
    out = np.zeros(s.shape)
    st = s.lib.st_dfdx_sym(s._h, F.ctypes.data, out.ctypes.data, 0, 1.0)
    assert st == ST_E_UNSUPPORTED
    Q = state(s.params)
    st = s.lib.st_species_rhs(s._h, Q.ctypes.data, np.zeros_like(Q).ctypes.data, out.ctypes.data,
                              out.ctypes.data)
    assert st == ST_E_UNSUPPORTED
    m = Solver(default_params(32))
    F = np.random.default_rng(0).standard_normal(m.shape)
    out = np.zeros(m.shape)
    assert m.lib.st_dfdx(m._h, F.ctypes.data, out.ctypes.data, 0, 1.0) == ST_E_UNSUPPORTED
    assert m.lib.st_rhs(m._h, ctypes.c_void_p(0), None, None) == -1
