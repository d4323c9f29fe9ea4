"""Serving loop: many blast-wave simulations of mixed grid sizes on one GPU.

Requests arrive over time (each one a full case: initial state, grid size,
number of LDDRK4 steps).  The server

  - admits a request when a solver slot of its grid size is free, or when a
    new slot fits in the HBM budget (first come, first served, with later
    requests allowed to start ahead of a head request that does not fit yet);
  - keeps every admitted case resident on the device in its own solver
    context (own CUDA stream), uploads its state once and reads back only the
    final state;
  - advances all admitted cases concurrently: each step is enqueued without
    waiting (from the third step on it is one CUDA-graph launch), so the
    cases' kernels overlap on the GPU, and a case that finishes frees its
    slot for the next request of that size while the others keep running;
  - records arrival, admission and completion times, from which p50/p99
    time-to-solution and aggregate cell-steps/s follow.

Slots are reused across requests of the same size (st_set_state resets a
context), so the scratch memory and captured step graph of a slot stay warm.
"""
import collections
import dataclasses
import time

import numpy as np

BYTES_PER_FIELD_ESTIMATE = 96       # fields of n^3 doubles per context before measurement


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


class _Slot:
    def __init__(self, n, solver, nbytes):
        self.n, self.solver, self.nbytes = n, solver, nbytes
        self.req = None
        self.step = 0
        self.admitted = 0.0


class Server:
    """make_solver(n) returns an object with set_state(Q, Y), set_time(t),
    setup(Q, Y) (the set-up before the main loop), step_async(step), done(),
    get_state() -> (Q, Y), get_time(), close() and memory_bytes(); the default
    builds a GPU solver context (Solver)."""

    def __init__(self, hbm_budget=150e9, make_solver=None, steps_ahead=2, clock=time.perf_counter, estimate=None,
                 max_active_cells=24e6):
        self.budget = float(hbm_budget)
        # cells of the cases stepped concurrently: enough to keep the GPU busy
        # with small cases, few enough that cases finish roughly in arrival
        # order instead of all sharing the GPU until the end
        self.max_active_cells = float(max_active_cells)
        self.make_solver = make_solver or _gpu_solver_factory()
        # bytes of one slot of grid n before a slot of that size has been measured
        self.estimate = estimate or (lambda n: BYTES_PER_FIELD_ESTIMATE * 8.0 * n ** 3)
        self.steps_ahead = max(1, int(steps_ahead))
        self.clock = clock
        self.slots = []                              # every context created
        self.free = collections.defaultdict(list)    # n -> idle slots
        self.footprint = {}                          # n -> measured bytes of one slot
        self.used = 0.0

    # -- memory accounting ------------------------------------------------------
    def _estimate(self, n):
        return self.footprint.get(n, self.estimate(n))

    def _evict_idle(self, keep_n, need):
        """Close idle slots of other sizes until `need` more bytes fit (only
        when closing them is enough)."""
        reclaimable = sum(sl.nbytes for n, lst in self.free.items() if n != keep_n for sl in lst)
        if self.used - reclaimable + need > self.budget:
            return
        for n in list(self.free):
            if n == keep_n:
                continue
            while self.free[n] and self.used + need > self.budget:
                slot = self.free[n].pop()
                slot.solver.close()
                self.slots.remove(slot)
                self.used -= slot.nbytes

    def _new_slot(self, n):
        solver = self.make_solver(n)
        nbytes = float(solver.memory_bytes())
        slot = _Slot(n, solver, nbytes)
        self.slots.append(slot)
        self.used += nbytes
        return slot

    def _try_admit(self, req, now):
        if self.free[req.n]:
            slot = self.free[req.n].pop()
        else:
            need = self._estimate(req.n)
            if self.used + need > self.budget:
                self._evict_idle(req.n, need)
            if self.used + need > self.budget:
                if not any(s.req is not None for s in self.slots) and need > self.budget:
                    raise ValueError(f"a {req.n}^3 case needs about {need:.3g} B, more than the HBM budget")
                return None
            slot = self._new_slot(req.n)
        slot.req = req
        slot.step = 0
        slot.admitted = now
        slot.solver.set_state(req.Q, req.Y)
        slot.solver.set_time(0.0)
        slot.solver.setup(req.Q, req.Y)
        return slot

    def _refresh_footprint(self, slot):
        # the scratch pool of a context grows during its first steps
        nb = float(slot.solver.memory_bytes())
        if nb > slot.nbytes:
            self.used += nb - slot.nbytes
            slot.nbytes = nb
        self.footprint[slot.n] = max(self.footprint.get(slot.n, 0.0), slot.nbytes)

    # -- main loop -------------------------------------------------------------
    def run(self, requests, idle_sleep=2e-4):
        """Serve the requests (arrival times relative to the call); returns the
        results in completion order."""
        pending = collections.deque(sorted(requests, key=lambda r: (r.arrival, r.rid)))
        waiting = []
        active = []
        results = []
        t0 = self.clock()
        while pending or waiting or active:
            now = self.clock() - t0
            while pending and pending[0].arrival <= now:
                waiting.append(pending.popleft())
            # admission: FIFO, later requests may pass a head that does not fit
            still = []
            active_cells = float(sum(sl.n ** 3 for sl in active))
            for req in waiting:
                if active and active_cells + req.n ** 3 > self.max_active_cells:
                    still.append(req)
                    continue
                slot = self._try_admit(req, now)
                if slot is not None:
                    active_cells += req.n ** 3
                if slot is None:
                    still.append(req)
                else:
                    active.append(slot)
            waiting = still
            progressed = False
            for slot in list(active):
                if not slot.solver.done():
                    continue
                progressed = True
                if slot.step > 0:
                    self._refresh_footprint(slot)
                if slot.step >= slot.req.steps:
                    Q, Y = slot.solver.get_state()
                    tsim = slot.solver.get_time()
                    done = self.clock() - t0
                    results.append(Result(slot.req.rid, slot.n, slot.req.steps, Q, Y, tsim, slot.req.arrival,
                                          slot.admitted, done))
                    slot.req = None
                    active.remove(slot)
                    self.free[slot.n].append(slot)
                    continue
                for _ in range(min(self.steps_ahead, slot.req.steps - slot.step)):
                    slot.solver.step_async(slot.step)
                    slot.step += 1
            if not progressed and (not pending or pending[0].arrival > self.clock() - t0):
                time.sleep(idle_sleep)
        return results

    def close(self):
        for slot in self.slots:
            slot.solver.close()
        self.slots.clear()
        self.free.clear()
        self.used = 0.0


def _gpu_solver_factory(**param_kw):
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

        def get_state(self, Q=None, Y=None):
            return Solver.get_state(self, Q, Y)

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
