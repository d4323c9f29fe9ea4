"""Serving loop on the GPU: cases of mixed grid sizes admitted while others
run, overlapping on the device, each result identical to the same case run
alone (same kernels, same order within a context; tolerance 1e-12)."""
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
    from shock_turbulence_b200.serving import Request, Server, _gpu_solver_factory, summarize
    steps = [5, 4, 6, 4, 5, 3]
    reqs = []
    for i, (n, k) in enumerate(zip(sizes, steps)):
        Q, Y = case(n, seed=10 + i, p_ratio=20.0 + 10 * i)
        reqs.append(Request(i, n, k, Q, Y, arrival=0.01 * i))
    srv = Server(hbm_budget=2e9, make_solver=_gpu_solver_factory(precision=precision))
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
