"""FP32 mode (float intermediates, double state, accumulators, state filter and
pressure recovery) against the FP64 path and the CPU oracle.

Tolerance: relative L2 error per conserved field <= 1e-5 after 100 steps
(the precision workload's horizon), the bound the FP32 mode is specified to; Linf is reported beside it
and bounded at 1e-4.  Single operators (one RHS evaluation, whose derivatives
of float-rounded fields carry an error of about eps_float * N) are bounded at
1e-4 relative L2."""
import ctypes

import numpy as np
import pytest

from shock_turbulence_b200.params import PRECISION_FP32, PRECISION_FP64, default_params, periodic_params
from shock_turbulence_b200.precision import field_errors, worst

pytestmark = pytest.mark.gpu

L2_TOL = 1e-5
LINF_TOL = 1e-4
NSTEPS = 100


def blast(p, seed=5):
    """Blast in turbulence with a mass-fraction front crossing the domain."""
    from shock_turbulence_b200.initial import blast_in_turbulence
    x = np.linspace(0, 1, p.nx)[:, None, None]
    y = np.linspace(0, 1, p.ny)[None, None, :]
    Yf = 0.5 + 0.5 * np.tanh(8 * (np.sqrt(x ** 2 + y ** 2) - 0.5)) * np.ones((p.nx, p.nz, p.ny))
    return blast_in_turbulence(p, k0=4, mach_t=0.1, p_ratio=100.0, radius_cells=4, seed=seed, y_field=Yf)


def run(p, Q, Y, nsteps):
    from shock_turbulence_b200 import Solver
    s = Solver(p)
    s.set_state(Q, Y)
    if p.family == 0:
        s.Compute_gamma(Y)
    s.Compute_hyper(Q, Y)
    t, k = 0.0, 0
    for _ in range(nsteps):
        t, k = s.step(t, k)
    Qo, Yo = s.get_state()
    s.close()
    return Qo, Yo, t


def report(errs):
    return ", ".join(f"{k} L2 {v[0]:.2e} Linf {v[1]:.2e}" for k, v in errs.items())


def test_blast_steps_vs_fp64():
    kw = dict(hyper_param=1, c_beta_scale=1.75)
    p64 = default_params(64, **kw)
    p32 = default_params(64, precision=PRECISION_FP32, **kw)
    Q, Y = blast(p64)
    Q64, Y64, t64 = run(p64, Q, Y, NSTEPS)
    Q32, Y32, t32 = run(p32, Q, Y, NSTEPS)
    errs = field_errors(Q32, Q64, Y32, Y64)
    l2, linf = worst(errs)
    print(f"blast 64^3, {NSTEPS} steps:", report(errs))
    assert np.isfinite(Q32).all()
    assert abs(t32 - t64) <= 1e-5 * t64
    assert l2 <= L2_TOL, report(errs)
    assert linf <= LINF_TOL, report(errs)


def test_periodic_steps_vs_fp64():
    from shock_turbulence_b200.initial import periodic_turbulence
    p64 = periodic_params(64)
    p32 = periodic_params(64, precision=PRECISION_FP32)
    Q = periodic_turbulence(p64, k0=4.0, urms=0.1, seed=2)
    Q64, _, t64 = run(p64, Q, None, NSTEPS)
    Q32, _, t32 = run(p32, Q, None, NSTEPS)
    errs = field_errors(Q32, Q64)
    l2, linf = worst(errs)
    print(f"periodic 64^3, {NSTEPS} steps:", report(errs))
    assert abs(t32 - t64) <= 1e-5 * t64
    assert l2 <= L2_TOL, report(errs)
    assert linf <= LINF_TOL, report(errs)


def test_steps_vs_oracle(oracle_mod):
    """FP32 GPU steps against the FP64 CPU oracle directly (100 steps)."""
    from shock_turbulence_b200 import Solver
    p = default_params(32, 32, 64, re=100.0, precision=PRECISION_FP32)
    po = default_params(32, 32, 64, re=100.0)
    s, o = Solver(p), oracle_mod.Oracle(po)
    Q, Y = blast(po, seed=7)
    for h in (s, o):
        h.set_state(Q, Y)
    s.Compute_gamma(Y); o.compute_gamma(Y)
    s.Compute_hyper(Q, Y); o.compute_hyper(Q, Y)
    ts, ss, to, so = 0.0, 0, 0.0, 0
    for _ in range(NSTEPS):
        ts, ss = s.step(ts, ss)
        to, so = o.step(to, so)
    Qg, Yg = s.get_state()
    Qo, Yo = o.get_state()
    errs = field_errors(Qg, Qo, Yg, Yo)
    print(f"oracle 32x32x64, {NSTEPS} steps:", report(errs))
    assert worst(errs)[0] <= L2_TOL, report(errs)


def test_rhs_operator_vs_fp64():
    """One RHS + Hyper_RHS evaluation through the per-operator entry points."""
    from shock_turbulence_b200 import Solver
    p64 = default_params(32, 64, 32, re=100.0)
    p32 = default_params(32, 64, 32, re=100.0, precision=PRECISION_FP32)
    Q, Y = blast(p64, seed=9)
    out = []
    for p in (p64, p32):
        s = Solver(p)
        s.set_state(Q, Y)
        s.Compute_gamma(Y)
        R = s.field(5)
        s.RHS(Q.copy(), R, Y)
        s.Hyper_RHS(Q, R, Y)
        out.append((R, s.get_common("visc_hyper"), s.get_common("dux_dx")))
        s.close()
    for l in range(5):
        e = np.linalg.norm(out[1][0][l] - out[0][0][l]) / np.linalg.norm(out[0][0][l])
        assert e <= 1e-4, (l, e)
    for k in (1, 2):
        e = np.linalg.norm(out[1][k] - out[0][k]) / np.linalg.norm(out[0][k])
        assert e <= 1e-4, (k, e)


def test_fp32_memory_smaller():
    from shock_turbulence_b200 import Solver
    b = []
    for prec in (PRECISION_FP64, PRECISION_FP32):
        s = Solver(default_params(32, precision=prec))
        v = ctypes.c_longlong()
        assert s.lib.st_memory(s._h, ctypes.byref(v)) == 0
        b.append(v.value)
        s.close()
    assert b[1] < b[0]


def test_bad_precision_rejected():
    from shock_turbulence_b200 import Solver, StError
    with pytest.raises(StError):
        Solver(default_params(32, precision=7))


def test_fp32_needs_32_lines():
    """The FP32 kernels give a CTA 32 lines (two per thread): ny must be a
    multiple of 32; 48 is rejected as unsupported, not run on another path."""
    from shock_turbulence_b200 import Solver, StError
    with pytest.raises(StError) as e:
        Solver(default_params(32, 48, 32, precision=PRECISION_FP32))
    assert e.value.status == -4
    Solver(default_params(32, 48, 32)).close()    # the FP64 path takes it
