"""Serving loop: many blast-wave simulations of mixed grid sizes on one GPU.

Requests arrive over time (each one a full case: initial state, grid size,
number of LDDRK4 steps).  The server

  - keeps one batch context per grid size (st_create_batch): its cases share
    every kernel launch of a step, so k same-size cases cost one launch per
    operator instead of k, and cases of different sizes overlap on the GPU
    through their batches' streams;
  - admits a request when its size's batch has a free case slot, or when a
    new batch fits in the HBM budget (first come, first served, with later
    requests allowed to start ahead of a head request that does not fit yet);
    a case joins a running batch between steps, at its own step 0, while the
    others continue (each case has its own time step, time and step count);
  - keeps every admitted case resident on the device, uploads its state once
    and reads back only its final state; a finished case's slot is refilled
    by moving the batch's last active case into it, so the active cases stay
    in front and every launch covers active cases only;
  - enqueues the steps of each batch without waiting (one CUDA-graph launch
    per step, one graph per active count), never past the first case to
    finish;
  - records arrival, admission and completion times, from which p50/p99
    time-to-solution and aggregate cell-steps/s follow.

A batch's capacity is the number of cases of its size that fit in
``batch_cells`` cells (at least one, at most ``max_batch``).  A case gives
the same bytes in a batch as alone: same kernels, same arithmetic per cell,
its own reductions and time step.
"""
import collections
import dataclasses
import time

import numpy as np

BYTES_PER_FIELD_ESTIMATE = 96       # fields of n^3 doubles per case before measurement


@dataclasses.dataclass
class Request:
    rid: int
    n: int                            # grid points per direction
    steps: int                        # LDDRK4 steps to run
    Q: np.ndarray                     # initial state (5, n, n, n)
    Y: np.ndarray                     # initial mass fraction (n, n, n)
    arrival: float = 0.0              # seconds after the start of the run


@dataclasses.dataclass
class Result:
    rid: int
    n: int
    steps: int
    Q: np.ndarray
    Y: np.ndarray
    time: float                       # simulated time reached
    arrival: float
    admitted: float
    done: float

    @property
    def latency(self):
        return self.done - self.arrival


class _Case:
    def __init__(self, req, admitted):
        self.req = req
        self.step = 0
        self.admitted = admitted


class _Group:
    """One batch context of grid size n and its cases (slot k <-> cases[k])."""

    def __init__(self, n, batch, capacity, nbytes):
        self.n, self.batch, self.capacity, self.nbytes = n, batch, capacity, nbytes
        self.cases = []

    @property
    def cells(self):
        return len(self.cases) * self.n ** 3


class Server:
    """make_batch(n, capacity) returns an object with start(k, Q, Y),
    set_active(na), get(k) -> (Q, Y, time, step), move(src, dst),
    step_async(), done(), memory_bytes() and close(); the default builds a
    GPU batch context (Batch)."""

    def __init__(self, hbm_budget=150e9, make_batch=None, steps_ahead=2, clock=time.perf_counter, estimate=None,
                 max_active_cells=24e6, batch_cells=16e6, max_batch=16):
        self.budget = float(hbm_budget)
        # cells of the cases stepped concurrently: enough to keep the GPU busy
        # with small cases, few enough that cases finish roughly in arrival
        # order instead of all sharing the GPU until the end
        self.max_active_cells = float(max_active_cells)
        self.batch_cells = float(batch_cells)
        self.max_batch = int(max_batch)
        self.make_batch = make_batch or _gpu_batch_factory()
        # bytes of one case of grid n before a batch of that size has been measured
        self.estimate = estimate or (lambda n: BYTES_PER_FIELD_ESTIMATE * 8.0 * n ** 3)
        self.steps_ahead = max(1, int(steps_ahead))
        self.clock = clock
        self.groups = {}                             # n -> _Group
        self.footprint = {}                          # n -> measured bytes per case
        self.used = 0.0

    # -- batches and memory ------------------------------------------------------
    def capacity(self, n):
        return int(max(1, min(self.max_batch, self.batch_cells // n ** 3)))

    def _per_case(self, n):
        return self.footprint.get(n, self.estimate(n))

    def _evict_idle(self, keep_n, need):
        """Close empty batches of other sizes until `need` more bytes fit (only
        when closing them is enough)."""
        idle = [g for n, g in self.groups.items() if n != keep_n and not g.cases]
        if self.used - sum(g.nbytes for g in idle) + need > self.budget:
            return
        for g in idle:
            if self.used + need <= self.budget:
                break
            g.batch.close()
            self.used -= g.nbytes
            del self.groups[g.n]

    def _group(self, n):
        g = self.groups.get(n)
        if g is not None:
            return g
        per = self._per_case(n)
        cap = self.capacity(n)
        if self.used + per * cap > self.budget:
            self._evict_idle(n, per)
        # as many case slots as the budget leaves room for, up to the capacity
        cap = min(cap, int((self.budget - self.used) // per)) if per > 0 else cap
        if cap < 1:
            busy = any(gr.cases for gr in self.groups.values())
            if not busy and per > self.budget:
                raise ValueError(f"a {n}^3 case needs about {per:.3g} B, more than the HBM budget")
            return None
        b = self.make_batch(n, cap)
        g = _Group(n, b, cap, float(b.memory_bytes()))
        self.groups[n] = g
        self.used += g.nbytes
        return g

    def _refresh_footprint(self, g):
        # the scratch pool of a context grows during its first steps
        nb = float(g.batch.memory_bytes())
        if nb > g.nbytes:
            self.used += nb - g.nbytes
            g.nbytes = nb
        self.footprint[g.n] = max(self.footprint.get(g.n, 0.0), g.nbytes / g.capacity)

    # -- main loop -------------------------------------------------------------
    def run(self, requests, idle_sleep=2e-4):
        """Serve the requests (arrival times relative to the call); returns the
        results in completion order."""
        pending = collections.deque(sorted(requests, key=lambda r: (r.arrival, r.rid)))
        waiting = []
        results = []
        t0 = self.clock()
        while pending or waiting or any(g.cases for g in self.groups.values()):
            now = self.clock() - t0
            while pending and pending[0].arrival <= now:
                waiting.append(pending.popleft())
            progressed = False
            # finished cases leave their batch (only between steps)
            for g in list(self.groups.values()):
                if not g.cases or not g.batch.done():
                    continue
                if any(cs.step > 0 for cs in g.cases):
                    self._refresh_footprint(g)
                k = 0
                while k < len(g.cases):
                    cs = g.cases[k]
                    if cs.step < cs.req.steps:
                        k += 1
                        continue
                    Q, Y, tsim, _ = g.batch.get(k)
                    done = self.clock() - t0
                    results.append(Result(cs.req.rid, g.n, cs.req.steps, Q, Y, tsim, cs.req.arrival,
                                          cs.admitted, done))
                    last = len(g.cases) - 1
                    if k != last:
                        g.batch.move(last, k)
                        g.cases[k] = g.cases[last]
                    g.cases.pop()
                    progressed = True
                if g.cases:
                    g.batch.set_active(len(g.cases))
            # admission: FIFO, later requests may pass a head that does not fit
            active_cells = float(sum(g.cells for g in self.groups.values()))
            still = []
            for req in waiting:
                if active_cells > 0 and active_cells + req.n ** 3 > self.max_active_cells:
                    still.append(req)
                    continue
                g = self._group(req.n)
                if g is None or len(g.cases) >= g.capacity or (g.cases and not g.batch.done()):
                    still.append(req)
                    continue
                k = len(g.cases)
                g.batch.start(k, req.Q, req.Y)
                g.cases.append(_Case(req, self.clock() - t0))
                g.batch.set_active(len(g.cases))
                active_cells += req.n ** 3
                progressed = True
            waiting = still
            # enqueue steps of every idle batch, never past its first finisher
            for g in self.groups.values():
                if not g.cases or not g.batch.done():
                    continue
                todo = min(self.steps_ahead, min(cs.req.steps - cs.step for cs in g.cases))
                for _ in range(todo):
                    g.batch.step_async()
                for cs in g.cases:
                    cs.step += todo
                progressed = progressed or todo > 0
            if not progressed and (not pending or pending[0].arrival > self.clock() - t0):
                time.sleep(idle_sleep)
        return results

    @property
    def slots(self):
        """Batch contexts currently held (one per grid size)."""
        return list(self.groups.values())

    def close(self):
        for g in self.groups.values():
            g.batch.close()
        self.groups.clear()
        self.used = 0.0


def _gpu_batch_factory(**param_kw):
    from . import Batch, default_params

    def make(n, capacity):
        kw = dict(re=100.0, re1=100.0, re2=100.0, pr=0.7, hyper_param=1, cfl_cal=0.5, c_beta_scale=1.75)
        kw.update(param_kw)
        return Batch(default_params(n, **kw), capacity)

    return make


def _gpu_solver_factory(**param_kw):
    """A single-grid solver with the serving parameters (for running a case alone)."""
    from . import Solver, default_params

    class _GpuSolver(Solver):
        def memory_bytes(self):
            import ctypes
            b = ctypes.c_longlong()
            self._check(self.lib.st_memory(self._h, ctypes.byref(b)), "st_memory")
            return b.value

        def setup(self, Q, Y):
            # the calls before the main loop, src/main_mf.f:100-104
            self.Compute_gamma(Y)
            self.Compute_hyper(Q, Y)

    def make(n):
        kw = dict(re=100.0, re1=100.0, re2=100.0, pr=0.7, hyper_param=1, cfl_cal=0.5, c_beta_scale=1.75)
        kw.update(param_kw)
        return _GpuSolver(default_params(n, **kw))

    return make


def summarize(results, t_total=None):
    """p50/p99 time-to-solution and aggregate Mcell-steps/s of a run."""
    lat = np.array([r.latency for r in results])
    work = float(sum(r.n ** 3 * r.steps for r in results))
    span = t_total if t_total is not None else max(r.done for r in results) - min(r.arrival for r in results)
    return {"requests": len(results), "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "makespan_s": float(span), "mcell_steps_per_s": work / span / 1e6}
