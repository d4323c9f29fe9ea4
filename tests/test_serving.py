"""Serving loop host logic on CPU with a fake batch: admission by HBM budget,
one batch per grid size, same-size cases stepped together (joining a running
batch at their own step 0, leaving it when done with the last active case
moved into the freed slot), FIFO with later requests passing a head that does
not fit, every request served with its own result."""
import numpy as np
import pytest

from shock_turbulence_b200.serving import Request, Server, summarize


class FakeBatch:
    """A step of the batch takes work proportional to its active cells on a
    shared clock; a case's state counts the steps it took."""
    created = []

    def __init__(self, n, capacity, clock):
        self.n, self.capacity, self.clock = n, capacity, clock
        self.Q = [None] * capacity
        self.Y = [None] * capacity
        self.steps = [0] * capacity
        self.active = 0
        self.busy_until = 0.0
        self.batch_steps = 0
        FakeBatch.created.append(self)

    def memory_bytes(self):
        return 10 * self.n ** 3 * self.capacity

    def start(self, k, Q, Y):
        assert self.done() and 0 <= k < self.capacity
        self.Q[k], self.Y[k] = Q.copy(), Y.copy()
        self.steps[k] = 0

    def set_active(self, na):
        assert 1 <= na <= self.capacity
        self.active = na

    def get(self, k):
        assert self.done()
        return self.Q[k], self.Y[k], float(self.steps[k]), self.steps[k]

    def move(self, src, dst):
        self.Q[dst], self.Y[dst], self.steps[dst] = self.Q[src], self.Y[src], self.steps[src]

    def step_async(self):
        start = max(self.busy_until, self.clock.now)
        self.busy_until = start + 1e-3 * self.n * self.active / 16
        for k in range(self.active):
            self.Q[k] = self.Q[k] + 1.0
            self.steps[k] += 1
        self.batch_steps += 1

    def done(self):
        return self.clock.now >= self.busy_until

    def close(self):
        pass


class Clock:
    def __init__(self):
        self.now = 0.0

    def __call__(self):
        self.now += 1e-4
        return self.now


def requests(sizes, steps, gap):
    steps = [steps] * len(sizes) if np.isscalar(steps) else steps
    return [Request(i, n, k, np.zeros((5, n, n, n)) + i, np.ones((n, n, n)), arrival=i * gap)
            for i, (n, k) in enumerate(zip(sizes, steps))]


def make_server(budget, **kw):
    clock = Clock()
    FakeBatch.created = []
    kw.setdefault("max_batch", 1)
    return Server(hbm_budget=budget, make_batch=lambda n, cap: FakeBatch(n, cap, clock), clock=clock,
                  estimate=lambda n: 10 * n ** 3, **kw), clock


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


def test_same_size_cases_share_a_batch():
    """Cases of one size with different step counts and arrival times run in
    one batch: a late case joins at its own step 0, finished cases leave
    (the last active case moves into the freed slot), every case takes
    exactly its own steps, and the batch steps fewer times than the cases do
    in total."""
    srv, _ = make_server(1e12, max_batch=4)
    steps = [7, 3, 5, 4, 6, 2]
    reqs = requests([16] * 6, steps=steps, gap=2e-3)
    res = srv.run(reqs, idle_sleep=0)
    assert sorted(r.rid for r in res) == list(range(6))
    for r in res:
        assert np.all(r.Q == r.rid + steps[r.rid]) and r.time == steps[r.rid]
    assert len(FakeBatch.created) == 1 and FakeBatch.created[0].capacity == 4
    assert FakeBatch.created[0].batch_steps < sum(steps)


def test_budget_limits_concurrency_and_batches_are_reused():
    # room for exactly one 32^3 batch (10 * 32^3 bytes) plus one 16^3 batch
    srv, _ = make_server(10 * 32 ** 3 + 10 * 16 ** 3)
    reqs = requests([32, 32, 32, 16, 16], steps=3, gap=0.0)
    res = srv.run(reqs, idle_sleep=0)
    assert sorted(r.rid for r in res) == list(range(5))
    sizes = sorted(b.n for b in FakeBatch.created)
    assert sizes == [16, 32]                      # one batch per size, reused
    assert srv.used <= srv.budget


def test_small_requests_pass_a_head_that_does_not_fit():
    srv, _ = make_server(10 * 48 ** 3 + 10 * 16 ** 3)
    reqs = requests([48, 48, 16], steps=4, gap=0.0)
    res = srv.run(reqs, idle_sleep=0)
    order = [r.rid for r in res]
    assert order.index(2) < order.index(1)       # the 16^3 case ran while the second 48^3 waited


def test_idle_batches_of_other_sizes_are_evicted():
    srv, _ = make_server(10 * 48 ** 3)
    reqs = requests([32, 48], steps=2, gap=0.05)
    res = srv.run(reqs, idle_sleep=0)
    assert sorted(r.rid for r in res) == [0, 1]
    assert [g.n for g in srv.slots] == [48]       # the idle 32^3 batch made room


def test_a_case_larger_than_the_budget_is_refused():
    srv, _ = make_server(10 * 16 ** 3)
    with pytest.raises(ValueError):
        srv.run(requests([32], steps=1, gap=0.0), idle_sleep=0)


def test_active_cell_cap_orders_completion():
    srv, _ = make_server(1e12, max_active_cells=2 * 16 ** 3, max_batch=4)
    res = srv.run(requests([16, 16, 16, 16], steps=3, gap=0.0), idle_sleep=0)
    done = {r.rid: r.done for r in res}
    assert max(done[0], done[1]) < min(done[2], done[3])
