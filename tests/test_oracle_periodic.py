"""Known-answer tests of the oracle's periodic single-fluid family
(src/derivCDopt6_periodic.f, src/filters_periodic.f, src/lddrk4_periodic_sf.f).

On a periodic grid a discrete Fourier mode is an eigenvector of every
constant-coefficient cyclic operator, so the compact derivatives, the compact
filter and the Gaussian filter must reproduce their modified wavenumbers /
transfer functions to rounding."""
import math

import numpy as np
import pytest

from conftest import rel_err

N = (32, 48, 16)   # nx, ny, nz


def params(**kw):
    from shock_turbulence_b200 import periodic_params
    return periodic_params(*N, **kw)


def mode(p, d, k):
    """sin(k * 2*pi*i/n) along direction d on the (Mx, Mz, My) array."""
    n = (p.nx, p.ny, p.nz)[d]
    t = 2 * math.pi * k * np.arange(n) / n
    shape = [1, 1, 1]
    axis = {0: 0, 1: 2, 2: 1}[d]
    shape[axis] = n
    base = np.broadcast_to(np.sin(t).reshape(shape), (p.nx, p.nz, p.ny))
    return np.ascontiguousarray(base), t.reshape(shape), axis, n


@pytest.mark.parametrize("d", [0, 1, 2])
@pytest.mark.parametrize("k", [1, 3, 7])
def test_first_derivative_modified_wavenumber(oracle_mod, d, k):
    p = params()
    o = oracle_mod.Oracle(p)
    F, t, axis, n = mode(p, d, k)
    out = np.zeros_like(F)
    o.dfd(d, 0, F, out, 0, 1.0)
    h = (p.x_leng, p.y_leng, p.z_leng)[d] / (n - 1)
    th = 2 * math.pi * k / n
    a, b, al = 14.0 / 9.0, 1.0 / 9.0, 1.0 / 3.0
    kmod = (a * math.sin(th) + 0.5 * b * math.sin(2 * th)) / (1 + 2 * al * math.cos(th)) / h
    expect = np.broadcast_to(kmod * np.cos(t), F.shape)
    assert rel_err(out, expect) < 1e-13


@pytest.mark.parametrize("d", [0, 1, 2])
@pytest.mark.parametrize("k", [1, 5])
def test_second_derivative_modified_wavenumber(oracle_mod, d, k):
    p = params()
    o = oracle_mod.Oracle(p)
    F, t, axis, n = mode(p, d, k)
    d1, out = np.zeros_like(F), np.zeros_like(F)
    o.d2fd2(d, 0, F, d1, out, 1)
    h = (p.x_leng, p.y_leng, p.z_leng)[d] / (n - 1)
    th = 2 * math.pi * k / n
    a2, b2, al = 12.0 / 11.0, 3.0 / 44.0, 2.0 / 11.0
    lam = -(2 * a2 * (1 - math.cos(th)) + 2 * b2 * (1 - math.cos(2 * th))) / (1 + 2 * al * math.cos(th)) / h ** 2
    assert rel_err(out, np.broadcast_to(lam * np.sin(t), F.shape)) < 1e-12
    ref = np.zeros_like(F)
    o.dfd(d, 0, F, ref, 0, 1.0)
    assert np.array_equal(d1, ref)        # iadd = 1 also returns the first derivative


@pytest.mark.parametrize("d", [0, 1, 2])
@pytest.mark.parametrize("k", [2, 6])
def test_filters_transfer_function(oracle_mod, d, k):
    p = params()
    o = oracle_mod.Oracle(p)
    F, t, axis, n = mode(p, d, k)
    th = 2 * math.pi * k / n
    a = [9.9965e-01, 0.66652, 0.16674, 4.0e-05, -5.0e-06]
    al, be = 6.6624e-01, 1.6688e-01
    T = (a[0] + 2 * sum(a[j] * math.cos(j * th) for j in range(1, 5))) / \
        (1 + 2 * al * math.cos(th) + 2 * be * math.cos(2 * th))
    out = np.zeros_like(F)
    o.filter(d, 0, F, out)
    assert rel_err(out, T * F) < 1e-12
    g = [float(np.float32(x)) for x in (3565 / 10368, 3091 / 12960, 1997 / 25920, 149 / 12960, 107 / 103680)]
    G = g[0] + 2 * sum(g[j] * math.cos(j * th) for j in range(1, 5))
    out = np.zeros_like(F)
    o.gauss(d, F, out)
    assert rel_err(out, G * F) < 1e-13


def _state(p, seed=3):
    from shock_turbulence_b200.initial import periodic_turbulence
    return periodic_turbulence(p, k0=4.0, urms=0.1, seed=seed)


def test_step_conserves_mass_and_is_finite(oracle_mod):
    p = params()
    o = oracle_mod.Oracle(p)
    Q = _state(p)
    o.set_state(Q, None)
    o.compute_hyper(Q)
    m0 = Q[3].mean()
    t, s = 0.0, 0
    for _ in range(2):
        t, s = o.step(t, s)
    Q1, _ = o.get_state()
    assert np.isfinite(Q1).all()
    assert abs(Q1[3].mean() - m0) < 1e-13 * m0
    mon = o.monitors()
    assert abs(mon[4] - Q1[3].mean()) < 1e-13
    assert t > 0 and s == 2
