"""Known-answer and property tests of the oracle's 1-D spherical-radial
family (src/derivCDopt6_radial.f, src/filters_nonperiodic.f,
src/rhsv_radial.f, src/hyper_radial.f, src/lddrk4_nonperiodic_sf.f)."""
import numpy as np
import pytest

from conftest import rel_err


@pytest.fixture(scope="module")
def rad(oracle_mod):
    from shock_turbulence_b200.params import radial_params
    return oracle_mod.Radial(radial_params())


def xcoord(n, x_leng):
    dx = x_leng / (n - 1)
    i = np.arange(1, n + 1)
    return ((i - n // 2) - 0.5) * dx


@pytest.mark.parametrize("n", [128, 201, 1000])
def test_radius_matches_reference_formula(rad, n):
    r = rad.radius(n, 2.0)
    assert np.allclose(r, np.abs(xcoord(n, 2.0)), rtol=0, atol=1e-15)
    assert r.min() > 0


@pytest.mark.parametrize("n", [128, 333])
def test_first_derivative_is_d_dr(rad, n):
    """Exact for quadratics in x on every row; d/dr = -d/dx on the left half."""
    x = xcoord(n, 2.0)
    F = x * x + 2.0 * x + 1.0
    out = np.zeros(n)
    rad.dfdx(2.0, F, out, 0, 1.0)
    expect = np.where(np.arange(1, n + 1) <= n // 2, -(2 * x + 2), 2 * x + 2)
    assert rel_err(out, expect) < 1e-12
    acc = np.ones(n)
    rad.dfdx(2.0, F, acc, 1, -0.5)
    assert rel_err(acc, 1.0 - 0.5 * expect) < 1e-12


@pytest.mark.parametrize("n", [128, 333])
def test_second_derivative_of_quadratic(rad, n):
    x = xcoord(n, 2.0)
    F = 3.0 * x * x - x
    d1, d2 = np.zeros(n), np.zeros(n)
    rad.d2fdx2(2.0, F, d1, d2, 1)
    assert rel_err(d2, np.full(n, 6.0)) < 1e-8     # 1/h^2 cancellation times the (1, 11) closure rows
    ref = np.zeros(n)
    rad.dfdx(2.0, F, ref, 0, 1.0)
    assert np.array_equal(d1, ref)


@pytest.mark.parametrize("n", [128, 777])
def test_filters_preserve_constants(rad, n):
    F = np.full(n, 2.5)
    out = np.zeros(n)
    rad.filter(F, out)
    assert np.abs(out - 2.5).max() < 1e-12
    g = np.zeros(n)
    rad.gauss(F, g)
    assert np.abs(g - 2.5).max() < 1e-6          # float32 coefficients sum to 1 within 1e-7


def test_rest_state_has_zero_rhs(rad):
    n = 256
    Q = np.zeros((3, n))
    Q[1] = 1.0
    Q[2] = 1.0 / 1.4
    R = np.zeros_like(Q)
    rad.rhs(2.0, Q, R)
    assert np.abs(R).max() < 1e-11


def test_blast_steps_stay_symmetric_and_finite(rad):
    from shock_turbulence_b200.initial import radial_blast
    n = 300
    Q = radial_blast(n, p_ratio=200.0, rng=np.random.default_rng(4))
    assert np.allclose(Q, Q[:, ::-1], rtol=0, atol=1e-14)
    hyp = np.zeros((2, n))
    rad.compute_hyper(2.0, Q, hyp)
    t, s = 0.0, 0
    for _ in range(3):
        dt, _, _ = rad.tstep(2.0, Q, hyp)
        assert dt > 0 and np.isfinite(dt)
        t, s = rad.step(2.0, Q, hyp, t, s)
    assert np.isfinite(Q).all() and s == 3 and t > 0
    assert rel_err(Q[:, ::-1], Q) < 1e-10
    assert Q[0, n // 2] > 0          # the blast drives u_r outward


def test_batch_equals_problem_by_problem(rad):
    from shock_turbulence_b200.initial import radial_batch
    lengths, xl, Q = radial_batch(5, nmin=128, nmax=300, seed=9)
    Qb = Q.copy()
    hyp = np.zeros(2 * lengths.sum())
    time = np.zeros(5)
    step = np.zeros(5, dtype=np.int32)
    rad.batch(lengths, xl, Qb, hyp, time, step, 2)
    off = 0
    for k, n in enumerate(lengths):
        q = Q[3 * off:3 * (off + n)].reshape(3, n).copy()
        h = np.zeros((2, n))
        rad.compute_hyper(xl[k], q, h)
        t, s = 0.0, 0
        for _ in range(2):
            t, s = rad.step(xl[k], q, h, t, s)
        assert np.array_equal(q.ravel(), Qb[3 * off:3 * (off + n)])
        assert t == time[k] and step[k] == 2
        off += n
