"""Output-side diagnostics on the GPU against the oracle: Compute_Grad
(src/grad_sym.f:13-120), Compute_SRM_Stats (pproc/pproc_mf.f:4-186) and
Generate_Shock_Surface (src/shock.f:163-260), on a blast state after two
LDDRK4 steps.  Sums are reduced in a different order than the reference's
sequential loops: tolerance 1e-12 relative (1e-11 for the fields, which go
through the compact derivatives)."""
import numpy as np
import pytest

from conftest import rel_err
from shock_turbulence_b200.params import PRECISION_FP32, default_params

pytestmark = pytest.mark.gpu


def blast(p, seed=8):
    from shock_turbulence_b200.initial import blast_in_turbulence
    x = np.linspace(0, 1, p.nx)[:, None, None]
    y = np.linspace(0, 1, p.ny)[None, None, :]
    Yf = 0.5 + 0.5 * np.tanh(8 * (np.sqrt(x ** 2 + y ** 2) - 0.5)) * np.ones((p.nx, p.nz, p.ny))
    return blast_in_turbulence(p, k0=4, mach_t=0.2, p_ratio=50.0, radius_cells=3, seed=seed, y_field=Yf)


@pytest.fixture(scope="module")
def pair(oracle_mod):
    from shock_turbulence_b200 import Solver
    p = default_params(32, 32, 64, re=100.0)
    s, o = Solver(p), oracle_mod.Oracle(p)
    Q, Y = blast(p)
    for h in (s, o):
        h.set_state(Q, Y)
    s.Compute_gamma(Y); o.compute_gamma(Y)
    s.Compute_hyper(Q, Y); o.compute_hyper(Q, Y)
    ts, ss, to, so = 0.0, 0, 0.0, 0
    for _ in range(2):
        ts, ss = s.step(ts, ss)
        to, so = o.step(to, so)
    return s, o


def test_compute_grad(pair):
    s, o = pair
    Gg, mg, eg = s.Compute_Grad()
    Go, mo, eo = o.compute_grad()
    for f in range(4):
        assert rel_err(Gg[f], Go[f]) < 1e-11, f
    assert mg == pytest.approx(mo, rel=1e-11)
    assert eg == pytest.approx(eo, rel=1e-11)
    # /GRAD/ left as the reference leaves it
    for name in ("duz_dy", "duy_dz", "dux_dx", "duz_dz"):
        assert rel_err(s.get_common(name), o.get_common(name)) < 1e-11, name


def test_srm_stats(pair):
    s, o = pair
    hg, tg, urg, yg = s.Compute_SRM_Stats()
    ho, to, uro, yo = o.compute_srm_stats()
    assert hg == pytest.approx(ho, rel=1e-12)
    assert tg == pytest.approx(to, rel=1e-12)
    assert np.allclose(urg, uro, rtol=1e-11, atol=1e-16, equal_nan=True)
    assert np.allclose(yg, yo, rtol=1e-12, equal_nan=True)


def test_shock_surface(pair):
    s, o = pair
    ag, bg = s.Generate_Shock_Surface()
    ao, bo = o.shock_surface()
    assert ag == pytest.approx(ao, rel=1e-12) and bg == pytest.approx(bo, rel=1e-12)
    assert ag > 0


def test_diagnostics_in_fp32_mode(pair):
    """The FP32 mode computes the diagnostics from its double state, with its
    float /HYPER/ beta widened: on the same state and beta they match the FP64
    context's (the shock surface to the float rounding of beta)."""
    from shock_turbulence_b200 import Solver
    s64, _ = pair
    Q, Y = s64.get_state()
    beta = s64.get_common("beta_hyper")
    s = Solver(default_params(32, 32, 64, re=100.0, precision=PRECISION_FP32))
    s.set_state(Q, Y)
    s.set_common("beta_hyper", beta)
    g32, g64 = s.Compute_Grad()[1:], s64.Compute_Grad()[1:]
    m32, m64 = s.Compute_SRM_Stats()[:2], s64.Compute_SRM_Stats()[:2]
    k32, k64 = s.Generate_Shock_Surface(), s64.Generate_Shock_Surface()
    s.close()
    assert g32 == pytest.approx(g64, rel=1e-12)
    assert m32 == pytest.approx(m64, rel=1e-12)
    assert k32 == pytest.approx(k64, rel=1e-3)
