"""Line operators and physics on an anisotropic grid against the CPU oracle,
through the C ABI.

The grid has a different length and spacing in each direction (x: 128
points over 2, y: 256 over 3, z: 192 over 1.5), so each direction runs a
different segmentation of the line solves (32 segments of 4, 8 and 6 rows)
with its own boundary closures, and every line operator is checked:
DF*/D2F*2 (sym and asym, iadd 0 and 1), Compact_Filter_* (out of place and
in place), the product forms inside RHS, Hyper_RHS and Species_RHS (the flux
derivatives read two to four fields) and a whole LDDRK4 step.  Tolerances:
1e-12 per line operator, 1e-11 per RHS field, 1e-10 for the artificial
viscosity and a whole step."""
import numpy as np
import pytest

from conftest import rel_err
from shock_turbulence_b200.params import default_params

pytestmark = pytest.mark.gpu
GRID = (128, 256, 192)          # (nx, ny, nz)
DIRS = "XYZ"


def params(**kw):
    p = default_params(*GRID, length=2.0, re=100.0, c_beta_scale=1.75, **kw)
    p.y_leng, p.z_leng = 3.0, 1.5
    return p


def field(shape, seed):
    nx, nz, ny = shape
    x = np.linspace(0, 1, nx)[:, None, None]
    z = np.linspace(0, 1, nz)[None, :, None]
    y = np.linspace(0, 1, ny)[None, None, :]
    f = np.sin(3 * x + 1) * np.cos(2 * y) * np.exp(z)
    return np.ascontiguousarray(f + 0.05 * np.random.default_rng(seed).standard_normal(shape))


def state(p, seed=5, p_ratio=50.0):
    from shock_turbulence_b200.initial import blast_in_turbulence
    x = np.linspace(0, 1, p.nx)[:, None, None]
    y = np.linspace(0, 1, p.ny)[None, None, :]
    Yf = 0.5 + 0.5 * np.tanh(8 * (np.sqrt(x ** 2 + y ** 2) - 0.5)) * np.ones((p.nx, p.nz, p.ny))
    return blast_in_turbulence(p, k0=4, mach_t=0.1, p_ratio=p_ratio, radius_cells=4, seed=seed, y_field=Yf)


@pytest.fixture(scope="module")
def pair(oracle_mod):
    from shock_turbulence_b200 import Solver
    p = params()
    s, o = Solver(p), oracle_mod.Oracle(p)
    yield s, o
    s.close()


@pytest.mark.parametrize("d", [0, 1, 2])
@pytest.mark.parametrize("asym", [0, 1])
def test_first_and_second_derivatives(pair, d, asym):
    s, o = pair
    sfx = "_asym" if asym else "_sym"
    F = field(s.shape, 10 + d + 3 * asym)
    for iadd, cadd in ((0, 1.0), (1, -0.5)):
        base = field(s.shape, 40 + d)
        g, r = base.copy(), base.copy()
        getattr(s, f"DFD{DIRS[d]}{sfx}")(F, g, iadd, cadd)
        o.dfd(d, asym, F, r, iadd, cadd)
        assert rel_err(g, r) < 1e-12, ("DFD", iadd)
        g1, g2, r1, r2 = (np.zeros(s.shape) for _ in range(4))
        getattr(s, f"D2FD{DIRS[d]}2{sfx}")(F, g1, g2, iadd)
        o.d2fd2(d, asym, F, r1, r2, iadd)
        assert rel_err(g2, r2) < 1e-12, ("D2FD2", iadd)
        if iadd:
            assert rel_err(g1, r1) < 1e-12


@pytest.mark.parametrize("d", [0, 1, 2])
@pytest.mark.parametrize("asym", [0, 1])
def test_compact_filters(pair, d, asym):
    s, o = pair
    sfx = "_asym" if asym else "_sym"
    F = field(s.shape, 60 + d + 3 * asym)
    g, r = np.zeros(s.shape), np.zeros(s.shape)
    getattr(s, f"Compact_Filter_{DIRS[d]}{sfx}")(F, g)
    o.filter(d, asym, F, r)
    assert rel_err(g, r) < 1e-12
    g = F.copy()
    getattr(s, f"Compact_Filter_{DIRS[d]}{sfx}")(g, g)      # F0 aliasing F
    assert rel_err(g, r) < 1e-12


def test_rhs_hyper_species(pair):
    """The flux derivatives of RHS (u*rho u_i, (rho E + P) u), Hyper_RHS
    (v_h S_ij, v_h S_ij u_i, k_h dT) and Species_RHS (rho u Y and the
    four-field diffusion forms) run as product forms of the line kernels."""
    s, o = pair
    Q, Y = state(s.params)
    for h in (s, o):
        h.set_state(Q, Y)
    s.Compute_gamma(Y)
    o.compute_gamma(Y)
    Qg, Qo = Q.copy(), Q.copy()
    Rg, Ro = np.zeros_like(Q), np.zeros_like(Q)
    s.RHS(Qg, Rg, Y)
    o.rhs(Qo, Ro, Y)
    for l in range(5):
        assert rel_err(Rg[l], Ro[l]) < 1e-11, ("RHS", l)
    s.Hyper_RHS(Qg, Rg, Y)
    o.hyper_rhs(Qo, Ro, Y)
    for name in ("beta_hyper", "visc_hyper", "k_hyper", "D_hyper"):
        assert rel_err(s.get_common(name), o.get_common(name)) < 1e-10, name
    for l in range(5):
        assert rel_err(Rg[l], Ro[l]) < 1e-10, ("Hyper_RHS", l)
    yg, yo = np.zeros_like(Y), np.zeros_like(Y)
    s.Species_RHS(Qg, Rg, Y, yg)
    o.species_rhs(Qo, Ro, Y, yo)
    assert rel_err(yg, yo) < 1e-10
    assert rel_err(Rg[4], Ro[4]) < 1e-10


def test_step(pair):
    s, o = pair
    Q, Y = state(s.params, seed=7, p_ratio=20.0)
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
