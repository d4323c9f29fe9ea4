"""GPU parity of the physics operators and of whole LDDRK4 steps against the
CPU oracle through the C ABI, on seeded blast-in-turbulence states with a
non-trivial mass fraction.  Tolerances: 1e-11 per operator (several line
solves compound), 1e-10 after full LDDRK4 steps."""
import numpy as np
import pytest

from conftest import rel_err
from shock_turbulence_b200.params import default_params

pytestmark = pytest.mark.gpu


def state(p, seed=3):
    from shock_turbulence_b200.initial import blast_in_turbulence
    nx, nz, ny = p.nx, p.nz, p.ny
    x = np.linspace(0, 1, nx)[:, None, None]
    y = np.linspace(0, 1, ny)[None, None, :]
    Yf = 0.5 + 0.5 * np.tanh(8 * (np.sqrt(x ** 2 + y ** 2 + 0 * x) - 0.5)) * np.ones((nx, nz, ny))
    return blast_in_turbulence(p, k0=4, mach_t=0.2, p_ratio=20.0, radius_cells=3, seed=seed, y_field=Yf)


@pytest.fixture(scope="module", params=[0.0, 100.0], ids=["re_gate_off", "re_gate_on"])
def setup(request, oracle_mod):
    from shock_turbulence_b200 import Solver
    p = default_params(32, 64, 32, re=request.param)
    s, o = Solver(p), oracle_mod.Oracle(p)
    Q, Y = state(p)
    for h in (s, o):
        h.set_state(Q, Y)
    s.Compute_gamma(Y)
    o.compute_gamma(Y)
    return s, o, Q, Y


def grads(h):
    names = ["dux_dx", "duy_dx", "duz_dx", "dux_dy", "duy_dy", "duz_dy", "dux_dz", "duy_dz", "duz_dz",
             "dTdx", "dTdy", "dTdz"]
    return {n: h.get_common(n) for n in names}


def test_compute_gamma(setup):
    s, o, Q, Y = setup
    assert rel_err(s.get_common("gamma_eff"), o.get_common("gamma_eff")) < 1e-14


def test_rhs(setup):
    s, o, Q, Y = setup
    Qg, Qo = Q.copy(), Q.copy()
    Rg, Ro = np.zeros_like(Q), np.zeros_like(Q)
    s.RHS(Qg, Rg, Y)
    o.rhs(Qo, Ro, Y)
    for l in range(5):
        assert rel_err(Rg[l], Ro[l]) < 1e-11, l
    assert rel_err(Qg, Qo) < 1e-15          # momenta rewritten as (m/rho)*rho
    gg, go = grads(s), grads(o)
    for k in gg:
        assert rel_err(gg[k], go[k]) < 1e-11, k


def test_hyper_species_bc_sponge(setup):
    s, o, Q, Y = setup
    Qg, Qo = Q.copy(), Q.copy()
    Rg, Ro = np.zeros_like(Q), np.zeros_like(Q)
    s.RHS(Qg, Rg, Y)
    o.rhs(Qo, Ro, Y)
    s.Hyper_RHS(Qg, Rg, Y)
    o.hyper_rhs(Qo, Ro, Y)
    for name in ("beta_hyper", "visc_hyper", "k_hyper", "D_hyper"):
        assert rel_err(s.get_common(name), o.get_common(name)) < 1e-10, name
    for l in range(5):
        assert rel_err(Rg[l], Ro[l]) < 1e-10, ("hyper", l)
    yg, yo = np.zeros_like(Y), np.zeros_like(Y)
    s.Species_RHS(Qg, Rg, Y, yg)
    o.species_rhs(Qo, Ro, Y, yo)
    assert rel_err(yg, yo) < 1e-10
    assert rel_err(Rg[4], Ro[4]) < 1e-10
    s.bc_RHS(Qg, Rg, Y, yg)
    o.bc_rhs(Qo, Ro, Y, yo)
    assert rel_err(Qg, Qo) < 1e-15
    for l in range(5):
        assert rel_err(Rg[l], Ro[l]) < 1e-10, ("bc", l)
    s.Sponge_Forcing(Qg, Rg, Y, yg)
    o.sponge_forcing(Qo, Ro, Y, yo)
    for l in range(5):
        assert rel_err(Rg[l], Ro[l]) < 1e-10, ("sponge", l)
    assert rel_err(yg, yo) < 1e-10


def test_fix_pressure_and_cfl(setup):
    s, o, Q, Y = setup
    Qg, Qo = Q.copy(), Q.copy()
    Qg[4, 3, 4, 5] = Qo[4, 3, 4, 5] = 0.0      # force one clipped cell
    s.Fix_Pressure(Qg, Y)
    o.fix_pressure(Qo, Y)
    assert rel_err(Qg, Qo) < 1e-15
    a = s.Compute_CFL(Q)
    b = o.compute_cfl(Q)
    assert abs(a[0] - b[0]) <= 1e-14 * b[0] and abs(a[1] - b[1]) <= 1e-14 * b[1]


@pytest.mark.parametrize("rk_mode", [0, 1])
def test_lddrk4_steps(oracle_mod, rk_mode):
    from shock_turbulence_b200 import Solver
    p = default_params(32, 32, 64, re=100.0, rk_mode=rk_mode)
    s, o = Solver(p), oracle_mod.Oracle(p)
    Q, Y = state(p, seed=7)
    for h in (s, o):
        h.set_state(Q, Y)
    s.Compute_gamma(Y); o.compute_gamma(Y)
    s.Compute_hyper(Q, Y); o.compute_hyper(Q, Y)
    ts, ss, to, so = 0.0, 0, 0.0, 0
    for _ in range(3):
        ts, ss = s.step(ts, ss)
        to, so = o.step(to, so)
    Qg, Yg = s.get_state()
    Qo, Yo = o.get_state()
    assert ss == so == 3
    assert abs(ts - to) <= 1e-12 * to
    for l in range(5):
        assert rel_err(Qg[l], Qo[l]) < 1e-10, l
    assert rel_err(Yg, Yo) < 1e-10
    mg, mo = s.monitors(), o.monitors()
    assert np.allclose(mg[:7], mo[:7], rtol=1e-10, atol=0)
