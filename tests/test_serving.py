"""Serving loop host logic on CPU with a fake solver: admission by HBM
budget, slot reuse per grid size, FIFO with later requests passing a head
that does not fit, every request served with its own result."""
import numpy as np
import pytest

from shock_turbulence_b200.serving import Request, Server, summarize


class FakeSolver:
    """Steps take 'work' ticks of a shared clock; state = step count."""
    created = []

    def __init__(self, n, clock):
        self.n, self.clock = n, clock
        self.Q = None
        self.busy_until = 0.0
        self.steps_done = 0
        FakeSolver.created.append(self)

    def memory_bytes(self):
        return 10 * self.n ** 3

    def set_state(self, Q, Y):
        self.Q, self.Y = Q.copy(), Y.copy()
        self.steps_done = 0

    def set_time(self, t):
        self.t = t

    def setup(self, Q, Y):
        pass

    def step_async(self, step):
        assert step == self.steps_done
        start = max(self.busy_until, self.clock.now)
        self.busy_until = start + 1e-3 * self.n / 16
        self.steps_done += 1
        self.Q = self.Q + 1.0

    def done(self):
        return self.clock.now >= self.busy_until

    def get_state(self):
        return self.Q, self.Y

    def get_time(self):
        return float(self.steps_done)

    def close(self):
        pass


class Clock:
    def __init__(self):
        self.now = 0.0

    def __call__(self):
        self.now += 1e-4
        return self.now


def requests(sizes, steps, gap):
    return [Request(i, n, steps, np.zeros((5, n, n, n)) + i, np.ones((n, n, n)), arrival=i * gap)
            for i, n in enumerate(sizes)]


def make_server(budget):
    clock = Clock()
    FakeSolver.created = []
    return Server(hbm_budget=budget, make_solver=lambda n: FakeSolver(n, clock), clock=clock,
                  estimate=lambda n: 10 * n ** 3), clock


pytestmark = pytest.mark.timeout(120)


def test_every_request_gets_its_own_result():
    srv, _ = make_server(1e12)
    reqs = requests([16, 32, 16, 48, 32], steps=5, gap=1e-3)
    res = srv.run(reqs, idle_sleep=0)
    assert sorted(r.rid for r in res) == list(range(5))
    for r in res:
        assert np.all(r.Q == r.rid + 5)           # initial value + one per step
        assert r.time == 5 and r.done >= r.admitted >= r.arrival
    s = summarize(res)
    assert s["requests"] == 5 and s["p99_s"] >= s["p50_s"] > 0


def test_budget_limits_concurrency_and_slots_are_reused():
    # room for exactly one 32^3 slot (10 * 32^3 bytes) plus one 16^3 slot
    srv, _ = make_server(10 * 32 ** 3 + 10 * 16 ** 3)
    reqs = requests([32, 32, 32, 16, 16], steps=3, gap=0.0)
    res = srv.run(reqs, idle_sleep=0)
    assert sorted(r.rid for r in res) == list(range(5))
    sizes = sorted(s.n for s in FakeSolver.created)
    assert sizes == [16, 32]                      # one slot per size, reused
    assert srv.used <= srv.budget


def test_small_requests_pass_a_head_that_does_not_fit():
    srv, _ = make_server(10 * 48 ** 3 + 10 * 16 ** 3)
    reqs = requests([48, 48, 16], steps=4, gap=0.0)
    res = srv.run(reqs, idle_sleep=0)
    order = [r.rid for r in res]
    assert order.index(2) < order.index(1)       # the 16^3 case ran while the second 48^3 waited


def test_idle_slots_of_other_sizes_are_evicted():
    srv, _ = make_server(10 * 48 ** 3)
    reqs = requests([32, 48], steps=2, gap=0.05)
    res = srv.run(reqs, idle_sleep=0)
    assert sorted(r.rid for r in res) == [0, 1]
    assert [s.n for s in srv.slots] == [48]       # the idle 32^3 slot made room


def test_a_case_larger_than_the_budget_is_refused():
    srv, _ = make_server(10 * 16 ** 3)
    with pytest.raises(ValueError):
        srv.run(requests([32], steps=1, gap=0.0), idle_sleep=0)


def test_active_cell_cap_orders_completion():
    clock = Clock()
    FakeSolver.created = []
    srv = Server(hbm_budget=1e12, make_solver=lambda n: FakeSolver(n, clock), clock=clock,
                 estimate=lambda n: 10 * n ** 3, max_active_cells=2 * 16 ** 3)
    res = srv.run(requests([16, 16, 16, 16], steps=3, gap=0.0), idle_sleep=0)
    assert len(FakeSolver.created) == 2            # at most two cases at a time, slots reused
    done = {r.rid: r.done for r in res}
    assert max(done[0], done[1]) < min(done[2], done[3])
