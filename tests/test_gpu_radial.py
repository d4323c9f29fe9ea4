"""Batched 1-D spherical-radial family on the GPU against the oracle
(src/derivCDopt6_radial.f, src/filters_nonperiodic.f, src/rhsv_radial.f,
src/hyper_radial.f, src/lddrk4_nonperiodic_sf.f).  Tolerances: 1e-12 per line
operator (relative to each problem's max), 1e-11 for RHS, 1e-10 for the
artificial viscosity and after full steps."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rad_oracle(oracle_mod):
    from shock_turbulence_b200.params import radial_params
    return oracle_mod.Radial(radial_params())


def batch(lengths, seed=7, params=None):
    from shock_turbulence_b200.initial import radial_blast
    from shock_turbulence_b200.radial import RadialBatch
    rng = np.random.default_rng(seed)
    lengths = np.asarray(lengths, dtype=np.int32)
    xl = np.full(len(lengths), 2.0)
    Q = np.concatenate([radial_blast(int(n), 2.0, float(rng.uniform(10, 1000)), rng=rng).ravel() for n in lengths])
    return RadialBatch(lengths, xl, params), Q


LENGTHS = [16, 37, 128, 500, 1024, 1025, 2047, 4096]


def per_problem(b, arr, nf):
    out, off = [], 0
    for n in b.lengths:
        out.append(arr[nf * off:nf * (off + n)])
        off += n
    return out


@pytest.mark.parametrize("op", ["d1", "d1add", "d2", "d2add", "filter", "gauss"])
def test_line_operators(rad_oracle, op):
    b, _ = batch(LENGTHS)
    F = np.random.default_rng(3).standard_normal(b.npts)
    G1, G2 = np.random.default_rng(4).standard_normal(b.npts), np.zeros(b.npts)
    R1, R2 = G1.copy(), np.zeros(b.npts)
    if op in ("d1", "d1add"):
        iadd = 1 if op == "d1add" else 0
        b.DFDX(F, G1, iadd, -0.5)
    elif op in ("d2", "d2add"):
        iadd = 1 if op == "d2add" else 0
        b.D2FDX2(F, G1 if iadd else None, G2, iadd)
    elif op == "filter":
        b.Compact_Filter_X(F, G1)
    else:
        b.Gaussian_Filter_X(F, G1)
    for k, (f, r1, r2) in enumerate(zip(per_problem(b, F, 1), per_problem(b, R1, 1), per_problem(b, R2, 1))):
        if op in ("d1", "d1add"):
            rad_oracle.dfdx(2.0, f, r1, iadd, -0.5)
        elif op in ("d2", "d2add"):
            rad_oracle.d2fdx2(2.0, f, r1, r2, iadd)
        elif op == "filter":
            rad_oracle.filter(f, r1)
        else:
            rad_oracle.gauss(f, r1)
    for k, (g, r) in enumerate(zip(per_problem(b, G1, 1), per_problem(b, R1, 1))):
        if op in ("d2",):
            continue
        assert rel_err(g, r) < 1e-12, (op, k, b.lengths[k])
    if op in ("d2", "d2add"):
        for k, (g, r) in enumerate(zip(per_problem(b, G2, 1), per_problem(b, R2, 1))):
            assert rel_err(g, r) < 1e-12, (op, k, b.lengths[k])


@pytest.mark.parametrize("hyper", [False, True])
def test_rhs(rad_oracle, hyper):
    b, Q = batch(LENGTHS, seed=11)
    G = np.zeros_like(Q)
    (b.RHS_with_hyper if hyper else b.RHS)(Q, G)
    off = 0
    for k, n in enumerate(b.lengths):
        q = Q[3 * off:3 * (off + n)].reshape(3, n)
        r = np.zeros((3, n))
        rad_oracle.rhs(2.0, q, r)
        if hyper:
            h = np.zeros((2, n))
            rad_oracle.hyper_rhs(2.0, q, r, h)
        g = G[3 * off:3 * (off + n)].reshape(3, n)
        for f in range(3):
            assert rel_err(g[f], r[f]) < (1e-10 if hyper else 1e-11), (k, n, f)
        off += n


@pytest.mark.parametrize("rk_mode", [0, 1])
def test_steps_match_oracle(rad_oracle, rk_mode):
    from shock_turbulence_b200.params import radial_params
    p = radial_params(rk_mode=rk_mode)
    b, Q = batch(LENGTHS, seed=5, params=p)
    b.set_state(Q)
    b.step(3)
    G = b.get_state()
    t, s = b.get_time()
    from oracle_py import Radial
    o = Radial(p)
    Qo = Q.copy()
    hyp = np.zeros(2 * b.npts)
    to = np.zeros(b.nprob)
    so = np.zeros(b.nprob, dtype=np.int32)
    o.batch(b.lengths, b.x_leng, Qo, hyp, to, so, 3)
    off = 0
    for k, n in enumerate(b.lengths):
        g = G[3 * off:3 * (off + n)].reshape(3, n)
        r = Qo[3 * off:3 * (off + n)].reshape(3, n)
        for f in range(3):
            scale = max(np.abs(r[f]).max(), 1e-300)
            assert np.abs(g[f] - r[f]).max() / scale < 1e-10, (k, n, f)
        off += n
    assert np.all(s == 3)
    assert np.abs(t - to).max() <= 1e-12 * to.max()


def test_every_configuration_and_tuner_agree(rad_oracle):
    b, Q = batch([64, 200, 1000, 1500, 3000], seed=2)
    ref = None
    for cs in range(3):
        for cl in range(3):
            b.config(cs, cl)
            b.set_state(Q)
            b.step(1)
            G = b.get_state()
            if ref is None:
                ref = G
            else:
                assert rel_err(G, ref) < 1e-12, (cs, cl)
    b.set_state(Q)
    (cs, cl), ms = b.tune()
    assert 0 <= cs <= 2 and 0 <= cl <= 2 and ms[0] > 0 and ms[1] > 0
    assert np.array_equal(b.get_state(), Q)          # tuning leaves the state alone
    b.step(1)
    assert rel_err(b.get_state(), ref) < 1e-12


def test_rejects_unsupported_lengths():
    from shock_turbulence_b200.radial import RadialBatch
    from shock_turbulence_b200.api import StError
    with pytest.raises(StError):
        RadialBatch([8], [2.0])
    with pytest.raises(StError):
        RadialBatch([5000], [2.0])


def test_100_steps_match_oracle():
    """100 steps of the reference's RK option (rk_mode 0), every problem
    against the oracle at 1e-10.  The 16-point problem is left out: with
    these pressure ratios the oracle itself overflows on it before step 100.
    The horizon is within what rounding allows: two oracle runs whose
    initial states differ by 1e-14 relative differ by at most 2.4e-11 after
    100 steps (5e-13 after 10; tests/oracle_sensitivity_radial.py).  The
    other RK option amplifies rounding faster (the same perturbation gives
    3e-11 after 10 steps and 5e-9 after 100), so it is held to the 3-step
    test above."""
    from shock_turbulence_b200.params import radial_params
    from oracle_py import Radial
    p = radial_params(rk_mode=0)
    b, Q = batch([37, 128, 500, 1024, 1025, 2047, 4096], seed=5, params=p)
    b.set_state(Q)
    b.step(100)
    G = b.get_state()
    t, s = b.get_time()
    o = Radial(p)
    Qo = Q.copy()
    hyp = np.zeros(2 * b.npts)
    to = np.zeros(b.nprob)
    so = np.zeros(b.nprob, dtype=np.int32)
    o.batch(b.lengths, b.x_leng, Qo, hyp, to, so, 100)
    assert np.isfinite(Qo).all()
    off = 0
    for k, n in enumerate(b.lengths):
        g = G[3 * off:3 * (off + n)].reshape(3, n)
        r = Qo[3 * off:3 * (off + n)].reshape(3, n)
        for f in range(3):
            assert np.abs(g[f] - r[f]).max() / np.abs(r[f]).max() < 1e-10, (k, n, f)
        off += n
    assert np.all(s == 100) and np.all(so == 100)
    assert np.abs(t - to).max() <= 1e-10 * to.max()
