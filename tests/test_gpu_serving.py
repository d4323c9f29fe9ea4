"""Serving loop and batch contexts on the GPU: cases of mixed grid sizes
admitted while others run, same-size cases stepped together in one batch
(one launch per operator for all of them), each result identical to the same
case run alone (same arithmetic per cell, its own reductions and time step:
the tests ask for the same bits, and at most 1e-12 in the mix)."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def case(n, seed, p_ratio):
    from shock_turbulence_b200.initial import blast_in_turbulence
    from shock_turbulence_b200.params import default_params
    p = default_params(n)
    return blast_in_turbulence(p, k0=4.0, mach_t=0.1, p_ratio=p_ratio, radius_cells=3.0, seed=seed)


def alone(n, Q, Y, steps, precision=0):
    from shock_turbulence_b200.serving import _gpu_solver_factory
    s = _gpu_solver_factory(precision=precision)(n)
    s.set_state(Q, Y)
    s.Compute_gamma(Y)
    s.Compute_hyper(Q, Y)
    t, st = 0.0, 0
    for _ in range(steps):
        t, st = s.step(t, st)
    out = s.get_state()
    s.close()
    return out, t


@pytest.mark.parametrize("precision,sizes", [(0, [32, 48, 32, 64, 48, 32]), (1, [32, 64, 32, 96, 64, 32])],
                         ids=["fp64", "fp32"])
def test_results_in_the_mix_equal_results_alone(precision, sizes):
    from shock_turbulence_b200.serving import Request, Server, _gpu_batch_factory, summarize
    steps = [5, 4, 6, 4, 5, 3]
    reqs = []
    for i, (n, k) in enumerate(zip(sizes, steps)):
        Q, Y = case(n, seed=10 + i, p_ratio=20.0 + 10 * i)
        reqs.append(Request(i, n, k, Q, Y, arrival=0.01 * i))
    srv = Server(hbm_budget=4e9, make_batch=_gpu_batch_factory(precision=precision))
    res = srv.run(reqs)
    srv.close()
    assert sorted(r.rid for r in res) == list(range(len(reqs)))
    for r in res:
        assert np.isfinite(r.Q).all()
        req = reqs[r.rid]
        (Qa, Ya), ta = alone(req.n, req.Q, req.Y, req.steps, precision)
        for f in range(5):
            assert rel_err(r.Q[f], Qa[f]) <= 1e-12, (r.rid, f)
        assert rel_err(r.Y, Ya) <= 1e-12
        assert abs(r.time - ta) <= 1e-12 * ta
    s = summarize(res)
    assert s["p99_s"] >= s["p50_s"] > 0 and s["mcell_steps_per_s"] > 0


def test_graph_step_equals_eager_step():
    from shock_turbulence_b200.serving import _gpu_solver_factory
    n = 32
    Q, Y = case(n, seed=3, p_ratio=50.0)
    s = _gpu_solver_factory()(n)
    s.set_state(Q, Y)
    s.set_time(0.0)
    s.setup(Q, Y)
    for k in range(6):
        s.step_async(k)                 # steps 2..5 replay the captured graph
    Qg, Yg = s.get_state()
    tg = s.get_time()
    s.close()
    (Qa, Ya), ta = alone(n, Q, Y, 6)
    assert np.array_equal(Qg, Qa) and np.array_equal(Yg, Ya) and tg == ta


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
def test_batch_cases_equal_cases_alone(precision):
    """Three 64^3 cases in one batch context: case 2 joins after two batch
    steps, case 0 leaves after four and case 2 moves into its slot; every
    case ends with the same bits as when run alone for its own steps."""
    from shock_turbulence_b200 import Batch
    from shock_turbulence_b200.params import default_params
    n = 64
    kw = dict(re=100.0, re1=100.0, re2=100.0, pr=0.7, hyper_param=1, cfl_cal=0.5, c_beta_scale=1.75)
    b = Batch(default_params(n, precision=precision, **kw), 3)
    cases = [case(n, seed=20 + i, p_ratio=30.0 + 20 * i) for i in range(3)]
    b.start(0, *cases[0])
    b.start(1, *cases[1])
    b.set_active(2)
    for _ in range(2):
        b.step_async()
    b.start(2, *cases[2])
    b.set_active(3)
    for _ in range(2):
        b.step_async()
    Q0, Y0, t0, s0 = b.get(0)                  # case 0: 4 steps
    b.move(2, 0)                               # case 2 (2 steps) into slot 0
    b.set_active(2)
    b.step_async()
    Q1, Y1, t1, s1 = b.get(1)                  # case 1: 5 steps
    Q2, Y2, t2, s2 = b.get(0)                  # case 2: 3 steps
    b.close()
    assert (s0, s1, s2) == (4, 5, 3)
    for (Qb, Yb, tb), i, k in (((Q0, Y0, t0), 0, 4), ((Q1, Y1, t1), 1, 5), ((Q2, Y2, t2), 2, 3)):
        (Qa, Ya), ta = alone(n, *cases[i], k, precision)
        assert np.array_equal(Qb, Qa) and np.array_equal(Yb, Ya), (i, float(np.abs(Qb - Qa).max()))
        assert tb == ta


def test_single_grid_calls_refuse_a_batch():
    from shock_turbulence_b200 import Batch
    from shock_turbulence_b200.params import default_params
    b = Batch(default_params(32), 2)
    Q, Y = case(32, seed=1, p_ratio=20.0)
    assert b.lib.st_set_state(b._h, Q.ctypes.data, Y.ctypes.data) == -4
    with pytest.raises(Exception):
        b.start(2, Q, Y)                       # case index out of range
    b.close()

