"""Whole main-loop steps over the long horizon: 100 steps of Compute_CFL +
Compute_Tstep + LDDRK4 (src/main_mf.f:137-143 with
src/lddrk4_nonperiodic_mf.f:428-541; src/main.f:129-136 with
src/lddrk4_periodic_sf.f:311-432) on the GPU against the CPU oracle, stepped
side by side from the same state.

Bound: <= 1e-10 normwise relative difference (max|a-b| / max|b|) per
conserved field and for Y after 100 steps, the same bound the short-horizon
step tests hold after 3, and the same for the simulated time (the sum of the
100 time steps, each set by a maximum over the state).  The per-call
differences of the segmented line solves (~1e-14) must not grow through a
shocked flow; the test records the difference at steps 1, 10, 25, 50 and
100 so a failure shows how it grew.  The cases use the reference build's
RK option (rk_mode 0), and one case the other option (rk_mode 1)."""
import numpy as np
import pytest

from conftest import rel_err
from shock_turbulence_b200.params import default_params, periodic_params

pytestmark = pytest.mark.gpu

TOL = 1e-10
NSTEPS = 100
CHECK = (1, 10, 25, 50, 100)


def mf_state(p, seed, p_ratio):
    """Blast in turbulence with a mass-fraction front crossing the domain."""
    from shock_turbulence_b200.initial import blast_in_turbulence
    x = np.linspace(0, 1, p.nx)[:, None, None]
    y = np.linspace(0, 1, p.ny)[None, None, :]
    Yf = 0.5 + 0.5 * np.tanh(8 * (np.sqrt(x ** 2 + y ** 2) - 0.5)) * np.ones((p.nx, p.nz, p.ny))
    return blast_in_turbulence(p, k0=4, mach_t=0.1, p_ratio=p_ratio, radius_cells=4, seed=seed, y_field=Yf)


def errors(s, o, with_y):
    Qg, Yg = s.get_state()
    Qo, Yo = o.get_state()
    e = [rel_err(Qg[l], Qo[l]) for l in range(5)]
    if with_y:
        e.append(rel_err(Yg, Yo))
    return e, Qg


def march(s, o, with_y):
    ts = to = 0.0
    ks = ko = 0
    hist = {}
    for k in range(1, NSTEPS + 1):
        ts, ks = s.step(ts, ks)
        to, ko = o.step(to, ko)
        if k in CHECK:
            e, Qg = errors(s, o, with_y)
            assert np.isfinite(Qg).all(), k
            hist[k] = max(e)
    assert ks == ko == NSTEPS
    assert abs(ts - to) <= TOL * to, (ts, to)
    e, _ = errors(s, o, with_y)
    growth = ", ".join(f"step {k}: {v:.2e}" for k, v in hist.items())
    print("max field difference by step:", growth)
    for i, v in enumerate(e):
        assert v <= TOL, (i, v, growth)
    return ts


# The 64^3 case uses a weaker blast.  With pressure ratio 100 on 64^3 the
# computation itself amplifies rounding by about 1e4 between steps 90 and
# 100: two oracle runs whose initial states differ by 1e-15 relative agree
# to 9e-13 up to step 90 and differ by 6e-9 (rho E) at step 100
# (tests/oracle_sensitivity.py), and the GPU run parts from the oracle in
# the same way (3e-12 at step 50, 2e-8 at step 100).  No implementation
# that does not repeat the reference's operation order bit for bit can
# meet 1e-10 there.
#
# The other RK option (rk_mode 1: the second five-stage loop reuses
# alpha1/beta1, so both loops of a step advance the state by a time step)
# is less robust on these blasts: on 32x64x32 the oracle itself overflows to
# NaN at step 72 with pressure ratio 100 and at step 99 with 20, so its
# 100-step case uses pressure ratio 5, which the oracle runs stably.
@pytest.mark.parametrize("grid,p_ratio,rk", [((32, 64, 32), 100.0, 0), ((64, 64, 64), 20.0, 0),
                                             ((32, 64, 32), 5.0, 1)], ids=["32x64x32", "64^3", "32x64x32-rk1"])
def test_mf_blast_100_steps(oracle_mod, grid, p_ratio, rk):
    """_mf octant: symmetry planes, sponge and outflow faces, two species,
    molecular viscosity on (Re 100), artificial viscosity with C_beta 1.75."""
    from shock_turbulence_b200 import Solver
    p = default_params(*grid, re=100.0, rk_mode=rk, c_beta_scale=1.75)
    s, o = Solver(p), oracle_mod.Oracle(p)
    Q, Y = mf_state(p, seed=11, p_ratio=p_ratio)
    for h in (s, o):
        h.set_state(Q, Y)
    s.Compute_gamma(Y); o.compute_gamma(Y)
    s.Compute_hyper(Q, Y); o.compute_hyper(Q, Y)
    march(s, o, with_y=True)
    mg, mo = s.monitors(), o.monitors()
    assert np.allclose(mg[:7], mo[:7], rtol=1e-10, atol=0)
    s.close()


def test_periodic_config0_100_steps(oracle_mod):
    """The 64^3 periodic decaying-turbulence case (k0 4, u_rms 0.1, Re 100,
    Pr 0.7, artificial viscosity on, CFL 0.5), 100 steps instead of 10."""
    from shock_turbulence_b200 import Solver
    from shock_turbulence_b200.initial import periodic_turbulence
    p = periodic_params(64, 64, 64, re=100.0, pr=0.7, cfl_cal=0.5)
    s, o = Solver(p), oracle_mod.Oracle(p)
    Q = periodic_turbulence(p, k0=4.0, urms=0.1, seed=0)
    s.set_state(Q)
    o.set_state(Q, None)
    s.Compute_hyper(Q)
    o.compute_hyper(Q)
    march(s, o, with_y=False)
    Qg, _ = s.get_state()
    assert abs(Qg[3].mean() - Q[3].mean()) < 1e-12     # mass is conserved (to rounding, 100 steps)
    s.close()
