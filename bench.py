"""Benchmark: Mcell-steps/s of the FP64 per-stage RHS + LDDRK4 path.

Workload: 384^3 octant blast wave in isotropic turbulence (symmetry planes at
x=y=z=0, non-reflecting outflow + sponge at the far faces), two-species
"_mf" physics with Y = 1, FP64.  One step = Compute_CFL + Compute_Tstep +
LDDRK4 (10 RHS stages, src/main_mf.f:137-143).  Inputs are seeded synthetic
fields (see shock_turbulence_b200/initial.py); there is no public dataset.

Multi-GPU: replicas only (one independent case per rank, no collective in
the data path); value = cells * steps of all ranks / max rank time.

--impl reference times the CPU oracle (plain-C restatement of the reference
path; the Fortran reference cannot be compiled in this image) on the host
cores, on a bounded sample grid of the same workload.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-steps/s (FP64 RHS+LDDRK4 step, 10 RK stages/step)"
UNIT = "Mcell-steps/s"


def make_params(n, device=0, precision=0):
    from shock_turbulence_b200 import default_params
    # config: Re = 100 with the molecular viscous term added (re > 0),
    # Pr = 0.7, artificial viscosity on, CFL 0.5, bulk coefficient scale 1.75
    return default_params(n, re=100.0, re1=100.0, re2=100.0, pr=0.7, hyper_param=1, cfl_cal=0.5,
                          c_beta_scale=1.75, device=device, precision=precision)


# Interface bytes per cell and RK stage of the reference's operator graph for
# the _mf blast step (Re > 0, artificial viscosity on): DF*/D2F*2 at 16 or 24
# B, filter and Gaussian passes at 16 B, the stage update at 40 B per
# variable.  Counted by the instrumented CPU oracle; tests/test_graph_bytes.py
# keeps this figure equal to that count.
GRAPH_BYTES_PER_CELL_STAGE = 2848.0
METRIC_FP32 = "Mcell-steps/s (FP32-mode RHS+LDDRK4 step, 10 RK stages/step)"


def make_state(p, seed):
    from shock_turbulence_b200.initial import blast_in_turbulence
    return blast_in_turbulence(p, k0=8.0, mach_t=0.1, p_ratio=100.0, radius_cells=4.0, seed=seed)


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.gpu_id)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def gpu_smi_id(dev):
    import torch
    props = torch.cuda.get_device_properties(dev)
    uid = getattr(props, "uuid", None)
    if uid is not None:
        s = str(uid)
        return s if s.startswith("GPU-") else "GPU-" + s
    return dev


# ---------------------------------------------------------------- CPU oracle
def oracle_rate(n, steps, warm, threads):
    """Mcell-steps/s of the CPU oracle on an n^3 sample (host cores)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py
    oracle_py.build()
    oracle_py.set_threads(threads)
    p = make_params(n)
    Q, Y = make_state(p, seed=1)
    o = oracle_py.Oracle(p)
    o.set_state(Q, Y)
    o.compute_gamma(Y)
    o.compute_hyper(Q, Y)
    t, s = 0.0, 0
    for _ in range(warm):
        t, s = o.step(t, s)
    t0 = time.perf_counter()
    for _ in range(steps):
        t, s = o.step(t, s)
    el = time.perf_counter() - t0
    return n ** 3 * steps / el / 1e6, el


def cpu_model():
    """The host CPU's model name (/proc/cpuinfo), for the baseline record."""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def single_core_rate(n=64, steps=2):
    """The CPU oracle on one host thread: a 64^3 sample of the same workload,
    1 warm-up + 2 timed steps (about 15 s)."""
    rate, el = oracle_rate(n, steps, 1, 1)
    return {"value": rate, "unit": UNIT, "cores": 1,
            "sample": f"CPU oracle, {n}^3 sample, 1 warm-up + {steps} timed steps ({el:.1f} s), 1 thread"}


def traffic_ratio(kernel):
    """DRAM read+write bytes over algorithmic bytes per launch of `kernel`, from
    the committed ncu capture (profiles/ncu_traffic.txt, a small grid): the
    launch's traffic at any grid is this ratio times its algorithmic bytes."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        parts = line.split()
        if len(parts) >= 6 and parts[0] == kernel and not line.startswith("#"):
            return float(parts[5])
    return None


def run_reference(args, rank):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    n = args.cpu_n
    rate, el = oracle_rate(n, args.steps, args.warmup, threads)
    sample = (f"CPU oracle (C restatement of the reference path), {n}^3 sample of the same workload, "
              f"{args.warmup} warm-up + {args.steps} timed steps, {threads} OpenMP threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded blast-in-turbulence)",
        "config": {"workload": f"blast wave in isotropic turbulence, octant, sample {n}^3 of 384^3",
                   "grid": n, "parallelism": "host OpenMP"},
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample,
                         "cpu_model": cpu_model()},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- radial batch
RAD_METRIC = "Mpoint-steps/s (FP64 batch of 1-D radial blasts, 11 RK stages/step)"
RAD_UNIT = "Mpoint-steps/s"
RAD_OPS = 143          # line operators per problem step (13 per stage x 11 stages)


def radial_oracle_rate(nprob, steps, threads, seed):
    """CPU oracle on a sample of problems drawn like the benchmark's."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import oracle_py
    from shock_turbulence_b200.initial import radial_batch
    from shock_turbulence_b200.params import radial_params
    oracle_py.build()
    oracle_py.set_threads(threads)
    L, X, Q = radial_batch(nprob, seed=seed)
    o = oracle_py.Radial(radial_params())
    hyp = np.zeros(2 * L.sum())
    tm = np.zeros(nprob)
    st = np.zeros(nprob, dtype=np.int32)
    o.batch(L, X, Q, hyp, tm, st, 1)                   # warm-up step (and the set-up Compute_hyper)
    t0 = time.perf_counter()
    o.batch(L, X, Q, hyp, tm, st, steps)
    el = time.perf_counter() - t0
    return float(L.sum()) * steps / el / 1e6, el, int(L.sum())


def run_radial(args, rank, world, local, dist):
    """The batching configuration: nprob independent 1-D spherical-radial blast
    problems, lengths uniform in [128, 4096], peak pressure ratios uniform in
    [10, 1000], 1% random-phase density perturbation; every problem advances
    args.steps LDDRK4 steps in one persistent launch per problem class."""
    threads = os.cpu_count() or 1
    if args.impl == "reference":
        if rank != 0:
            return
        rate, el, pts = radial_oracle_rate(512, 10, threads, seed=3)
        sample = (f"CPU oracle (C restatement), 512 problems of the same distribution ({pts} points), "
                  f"1 warm-up + 10 timed steps, {threads} OpenMP threads")
        print(json.dumps({
            "impl": "reference", "metric": RAD_METRIC, "value": rate, "unit": RAD_UNIT, "n_gpus": args.gpus,
            "steps": 10, "warmup": 1, "ms_per_step": el / 10 * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded radial blasts)",
            "config": {"workload": "batch of 1-D radial blasts, sample of 512 problems", "parallelism": "host OpenMP"},
            "cpu_baseline": {"value": rate, "unit": RAD_UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": rate, "unit": RAD_UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
            flush=True)
        return
    import numpy as np
    import torch
    from shock_turbulence_b200.initial import radial_batch
    from shock_turbulence_b200.params import radial_params
    from shock_turbulence_b200.radial import RadialBatch
    from shock_turbulence_b200.replicas import aggregate_rate, max_over_ranks, replica_seed
    torch.cuda.set_device(local)
    L, X, Q = radial_batch(args.nprob, seed=replica_seed(2, rank))
    npts = int(L.sum())
    b = RadialBatch(L, X, radial_params(device=local))
    stream = torch.cuda.Stream()             # a real stream handle: 0 would select the batch's own stream
    b.set_stream(stream.cuda_stream)
    b.set_state(Q)
    b.step(1)                                           # set-up Compute_hyper + first step
    cfg, tune_ms = b.tune()
    if args.warmup > 1:
        b.step(args.warmup - 1)
    c0 = b.launch_count()
    clocks = ClockSampler(gpu_smi_id(local))

    def barrier():
        if dist is not None:
            dist.barrier()

    barrier()
    torch.cuda.synchronize()
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    b.step_async(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), dist, "cuda")
    launches = b.launch_count() - c0
    value = aggregate_rate(npts, args.steps, ms, world)
    G = b.get_state()
    t, st = b.get_time()
    finite = bool(np.isfinite(G).all())
    # end to end: pinned host state in, steps, state out
    e2e = None
    if args.e2e_steps > 0:
        Qh = torch.from_numpy(np.ascontiguousarray(G)).pin_memory()
        barrier()
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        b.set_state(Qh)
        b.step_async(args.e2e_steps)
        b.get_state(Qh)
        f1.record(stream)
        torch.cuda.synchronize()
        ms_e2e = max_over_ranks(f0.elapsed_time(f1), dist, "cuda")
        e2e = {"value": aggregate_rate(npts, args.e2e_steps, ms_e2e, world), "unit": RAD_UNIT,
               "h2d_bytes_per_step": 3 * npts * 8 / args.e2e_steps, "d2h_bytes_per_step": 3 * npts * 8 / args.e2e_steps,
               "steps": args.e2e_steps, "note": "one state upload and download around the timed steps"}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        rate, el, pts = radial_oracle_rate(512, 10, threads, seed=3)
        cpu = {"value": rate, "unit": RAD_UNIT, "cores": threads, "kind": "port",
               "sample": f"CPU oracle, 512 problems of the same distribution ({pts} points), 1 warm-up + 10 timed "
                         f"steps ({el:.1f} s), {threads} OpenMP threads", "cpu_model": cpu_model()}
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak = float(json.load(open(peaks_path))["hbm_gbs"]) if os.path.exists(peaks_path) else 6650.0
    alg = RAD_OPS * 16.0 * npts * args.steps          # every line operator: one field in, one out
    achieved = alg / (ms / 1e3) / 1e9
    if rank == 0:
        print(json.dumps({
            "metric": RAD_METRIC, "value": value, "unit": RAD_UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded radial blasts)",
            "config": {"workload": f"{args.nprob} independent 1-D spherical-radial blasts, n uniform in [128, 4096], "
                                   "pressure ratio uniform in [10, 1000], 1% density perturbation",
                       "points": npts, "kernel_config": {"short": cfg[0], "long": cfg[1]},
                       "tune_ms": tune_ms, "parallelism": f"replicas x{world}",
                       "l2": "state 207 MB per field set, larger than L2", "finite": finite,
                       "steps_done_min": int(st.min()),
                       "rk_stages_per_step": 11, "mpoint_stages_per_s": value * 11},
            "e2e": e2e, "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "kernel": "k_rad_steps", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "note": "line-operator interface bytes (16 B/point/operator, 143 operators per step); "
                                 "the operators run from shared memory and L2, so the kernel is latency-bound"},
            "cpu_baseline": cpu, "clocks": clk}), flush=True)
    b.close()


# ---------------------------------------------------------------- serving
SRV_SIZES = (64, 96, 128, 192, 256)
SRV_WEIGHTS = (0.3, 0.25, 0.2, 0.15, 0.1)


def serving_requests(nreq, steps, rate, seed):
    """Seeded Poisson stream: grid size by the weights above, blast pressure
    ratio uniform in [10, 200], seeded turbulence (k0 = 8, M_t = 0.1)."""
    import numpy as np
    from shock_turbulence_b200 import default_params
    from shock_turbulence_b200.initial import blast_in_turbulence
    from shock_turbulence_b200.serving import Request
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(nreq):
        t += rng.exponential(1.0 / rate)
        n = int(rng.choice(SRV_SIZES, p=SRV_WEIGHTS))
        pr = float(rng.uniform(10.0, 200.0))
        Q, Y = blast_in_turbulence(default_params(n), k0=8.0, mach_t=0.1, p_ratio=pr, radius_cells=4.0,
                                   seed=int(rng.integers(1 << 30)))
        out.append(Request(i, n, steps, Q, Y, arrival=t))
    return out


def run_serving(args, rank, world, local, dist):
    """The serving configuration: Poisson arrivals (20 requests/s) of blast
    cases of mixed grid sizes, 100 LDDRK4 steps each, admitted by a 150 GB HBM
    budget, device-resident, stepped concurrently (one stream and one graph
    per slot).  value = aggregate cell-steps/s over the run's makespan."""
    steps = args.steps if "--steps" in sys.argv else 100
    if args.impl == "reference":
        if rank != 0:
            return
        threads = os.cpu_count() or 1
        rate, el = oracle_rate(64, 2, 1, threads)
        print(json.dumps({
            "impl": "reference", "metric": "Mcell-steps/s (serving: mixed-size blast cases)", "value": rate,
            "unit": UNIT, "n_gpus": args.gpus, "steps": 2, "warmup": 1, "ms_per_step": el / 2 * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": "CPU oracle on a 64^3 case of the stream (one case at a time)"},
            "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"64^3 case, 1 warm-up + 2 steps, {threads} OpenMP threads"},
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}), flush=True)
        return
    import torch
    from shock_turbulence_b200.serving import Server, summarize
    torch.cuda.set_device(local)
    reqs = serving_requests(args.requests, steps, 20.0, seed=4 + rank)
    fp32 = args.precision == "fp32"
    from shock_turbulence_b200.serving import _gpu_batch_factory
    srv = Server(hbm_budget=150e9, make_batch=_gpu_batch_factory(precision=1 if fp32 else 0))
    # warm the slot kinds once (not timed): context creation, scratch pools, graphs
    clocks = ClockSampler(gpu_smi_id(local))
    clocks.start()
    t0 = time.perf_counter()
    res = srv.run(reqs)
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    summ = summarize(res)
    rate = max_over = summ["mcell_steps_per_s"]
    if dist is not None:
        from shock_turbulence_b200.replicas import max_over_ranks
        max_over = max_over_ranks(summ["makespan_s"], dist, "cuda")
        rate = world * sum(r.n ** 3 * r.steps for r in res) / max_over / 1e6
    h2d = sum(6 * r.n ** 3 * 8 for r in res)
    if rank == 0:
        print(json.dumps({
            "metric": "Mcell-steps/s (serving: mixed-size blast cases, 100 LDDRK4 steps each)", "value": rate,
            "unit": UNIT, "n_gpus": world, "steps": steps, "warmup": 0, "ms_per_step": None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 intermediates / f64 state" if fp32 else "f64",
            "data": "synthetic (seeded blast-in-turbulence requests)",
            "config": {"workload": f"{args.requests} requests, Poisson arrivals at 20/s, grid sizes {SRV_SIZES} with "
                                   f"weights {SRV_WEIGHTS}, pressure ratio uniform in [10, 200], 150 GB HBM budget",
                       "p50_s": summ["p50_s"], "p99_s": summ["p99_s"], "mean_s": summ["mean_s"],
                       "makespan_s": summ["makespan_s"], "batches": {g.n: g.capacity for g in srv.slots},
                       "sizes": [r.n for r in sorted(res, key=lambda r: r.rid)]},
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": h2d / max(1, steps * len(res)),
                    "d2h_bytes_per_step": h2d / max(1, steps * len(res)),
                    "note": "time to solution includes each case's state upload and final download"},
            "gpu_launches": None, "roofline": None, "cpu_baseline": None, "clocks": clk,
            "wall_s": wall}), flush=True)
    srv.close()


# ---------------------------------------------------------------- precision
def run_precision(args, rank, world, local, dist):
    """The precision configuration: the 384^3 blast case and a 512^3 periodic
    turbulence box, each run in FP64 and in the FP32 mode from the same
    initial state for `steps` steps (default 100); reports relative L2 and
    Linf error per conserved field and the FP32/FP64 speed of each."""
    steps = args.steps if "--steps" in sys.argv else 100
    if args.impl == "reference" or rank != 0:
        if args.impl == "reference" and rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the precision workload compares two GPU runs; "
                                                                 "the CPU reference arm is the blast3d workload"}))
        return
    import torch
    from shock_turbulence_b200 import PRECISION_FP32, PRECISION_FP64, Solver, periodic_params
    from shock_turbulence_b200.initial import periodic_turbulence
    from shock_turbulence_b200.precision import field_errors, worst
    torch.cuda.set_device(local)
    cases = []
    n_blast = args.n
    n_per = args.periodic_n
    cases.append(("blast", n_blast, lambda prec: make_params(n_blast, device=local, precision=prec),
                  lambda p: make_state(p, seed=1)))
    cases.append(("periodic", n_per, lambda prec: periodic_params(n_per, device=local, precision=prec),
                  lambda p: (periodic_turbulence(p, k0=8.0, urms=0.1, seed=3), None)))
    out = {}
    clocks = ClockSampler(gpu_smi_id(local))
    clocks.start()
    for name, n, mk, init in cases:
        p64 = mk(PRECISION_FP64)
        Q0, Y0 = init(p64)
        res = {}
        for prec in (PRECISION_FP64, PRECISION_FP32):
            p = mk(prec)
            s = Solver(p)
            stream = torch.cuda.current_stream()
            s._check(s.lib.st_set_stream(s._h, stream.cuda_stream), "st_set_stream")
            s.set_state(Q0, Y0 if name == "blast" else None)
            if name == "blast":
                s.Compute_gamma(Y0)
            s.Compute_hyper(Q0, Y0 if name == "blast" else None)
            t, k = 0.0, 0
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                t, k = s.step(t, k)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            Q, Y = s.get_state()
            res[prec] = (Q, Y, t, ms)
            s.close()
            del s
        Q64, Y64, t64, ms64 = res[PRECISION_FP64]
        Q32, Y32, t32, ms32 = res[PRECISION_FP32]
        errs = field_errors(Q32, Q64, Y32 if name == "blast" else None, Y64 if name == "blast" else None)
        l2, linf = worst(errs)
        out[name] = {"grid": n, "steps": steps, "fp64_ms_per_step": ms64 / steps, "fp32_ms_per_step": ms32 / steps,
                     "fp64_mcell_steps_per_s": n ** 3 * steps / (ms64 / 1e3) / 1e6,
                     "fp32_mcell_steps_per_s": n ** 3 * steps / (ms32 / 1e3) / 1e6,
                     "speedup_fp32": ms64 / ms32, "time_fp64": t64, "time_fp32": t32,
                     "errors": {k: {"l2_rel": v[0], "linf_rel": v[1]} for k, v in errs.items()},
                     "worst_l2_rel": l2, "worst_linf_rel": linf}
        del Q0, Y0, res
    clk = clocks.stop()
    b = out["blast"]
    print(json.dumps({
        "metric": METRIC_FP32, "value": b["fp32_mcell_steps_per_s"], "unit": UNIT, "n_gpus": 1, "steps": steps,
        "warmup": 0, "ms_per_step": b["fp32_ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 intermediates / f64 state", "data": "synthetic",
        "config": {"workload": f"precision: {n_blast}^3 blast and {n_per}^3 periodic box, FP64 and FP32-mode runs "
                               f"from the same state, {steps} steps each; relative L2/Linf per conserved field",
                   "cases": out},
        "clocks": clk}), flush=True)


# ---------------------------------------------------------------- kernel timing
def kernel_profile(s):
    """Per-kernel launches, device ms and algorithmic bytes recorded while the
    context's profiling was on; pointwise launches are folded into one entry
    and also returned per source site."""
    import ctypes
    buf = ctypes.create_string_buffer(1 << 16)
    s._check(s.lib.st_profile_report(s._h, buf, len(buf)), "st_profile_report")
    prof, sites = {}, {}
    for k, v in json.loads(buf.value.decode()).items():
        key = "k_pointwise" if k.startswith("k_pointwise@") else k
        if key != k:
            sites[k.split("@")[1]] = v
        a = prof.setdefault(key, {"launches": 0, "ms": 0.0, "bytes": 0.0})
        for f in ("launches", "ms", "bytes"):
            a[f] += v[f]
    return prof, sites


def kernel_table(prof, ms_total, steps):
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak = float(json.load(open(peaks_path))["hbm_gbs"]) if os.path.exists(peaks_path) else 6650.0
    tot = sum(v["ms"] for v in prof.values()) or 1.0
    out = {}
    for k, v in sorted(prof.items(), key=lambda kv: -kv[1]["ms"]):
        gbs = v["bytes"] / (v["ms"] / 1e3) / 1e9 if v["bytes"] and v["ms"] else None
        out[k] = {"launches": v["launches"], "ms_per_step": round(v["ms"] / steps, 3), "share": round(v["ms"] / tot, 4),
                  "GB/s": gbs, "frac": round(gbs / peak, 3) if gbs else None}
    return out


def top_sites(sites, n=12):
    return {"st_physics.cu:" + k: round(v["ms"], 2) for k, v in sorted(sites.items(), key=lambda kv: -kv[1]["ms"])[:n]}


# ---------------------------------------------------------------- extensions
def fp32_extension(args, local, Q0, Y0, ref_state, fp64_value):
    """The FP32 mode on the same 384^3 blast: the same warm-up and timed steps
    from the same initial state as the FP64 line, device-timed, and the
    relative L2/Linf error per field of its final state against the FP64
    run's."""
    import torch
    from shock_turbulence_b200 import Solver
    from shock_turbulence_b200.precision import field_errors, worst
    p = make_params(args.n, device=local, precision=1)
    s = Solver(p)
    stream = torch.cuda.current_stream()
    s._check(s.lib.st_set_stream(s._h, stream.cuda_stream), "st_set_stream")
    s.set_state(Q0, Y0)
    s.Compute_gamma(Y0)
    s.Compute_hyper(Q0, Y0)
    t, st = 0.0, 0
    for _ in range(args.warmup):
        t, st = s.step(t, st)
    torch.cuda.synchronize()
    clocks = ClockSampler(gpu_smi_id(local))
    s.lib.st_profile(s._h, 1)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        t, st = s.step(t, st)
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    s.lib.st_profile(s._h, 0)
    ms = e0.elapsed_time(e1)
    prof, sites = kernel_profile(s)
    Q32, Y32 = s.get_state()
    s.close()
    errs = field_errors(Q32, ref_state[0], Y32, ref_state[1])
    l2, linf = worst(errs)
    value = args.n ** 3 * args.steps / (ms / 1e3) / 1e6
    return {"metric": METRIC_FP32, "value": value, "unit": UNIT, "ms_per_step": ms / args.steps,
            "steps": args.steps, "warmup": args.warmup, "speedup_vs_fp64": value / fp64_value,
            "dtype": "f32 intermediates / f64 state, accumulators, state filter, pressure recovery",
            "errors_vs_fp64_after_steps": args.warmup + args.steps,
            "errors": {k: {"l2_rel": v[0], "linf_rel": v[1]} for k, v in errs.items()},
            "worst_l2_rel": l2, "worst_linf_rel": linf, "clocks": clk,
            "kernels": kernel_table(prof, ms, args.steps), "pointwise_sites_ms": top_sites(sites)}


def serving_extension(args, local, fp64_value):
    """A short serving run (FP32 mode): Poisson arrivals at 20/s of blast
    cases of mixed grid sizes, 100 LDDRK4 steps each, 150 GB HBM budget,
    same-size cases stepped together; aggregate cell-steps/s over the
    makespan and p50/p99 time to solution."""
    import torch
    from shock_turbulence_b200.serving import Server, _gpu_batch_factory, summarize
    torch.cuda.set_device(local)
    reqs = serving_requests(args.ext_requests, 100, 20.0, seed=4)
    srv = Server(hbm_budget=150e9, make_batch=_gpu_batch_factory(precision=1))
    clocks = ClockSampler(gpu_smi_id(local))
    clocks.start()
    res = srv.run(reqs)
    clk = clocks.stop()
    batches = {g.n: g.capacity for g in srv.slots}
    srv.close()
    summ = summarize(res)
    return {"metric": "Mcell-steps/s (serving: mixed-size blast cases, FP32 mode, 100 LDDRK4 steps each)",
            "value": summ["mcell_steps_per_s"], "unit": UNIT, "ratio_vs_fp64_plain": summ["mcell_steps_per_s"] / fp64_value,
            "requests": len(res), "p50_s": summ["p50_s"], "p99_s": summ["p99_s"], "makespan_s": summ["makespan_s"],
            "sizes": sorted(r.n for r in res), "batch_capacity": batches, "clocks": clk,
            "timing": "wall clock over the run (arrival of the first request to completion of the last)"}


# ---------------------------------------------------------------- GPU arm
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=384, help="grid points per direction")
    ap.add_argument("--cpu-n", type=int, default=96, help="grid of the CPU-oracle sample")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extensions", action="store_true",
                    help="blast3d, FP64, one GPU: skip the FP32-mode and serving measurements that the "
                         "default line carries under 'extensions'")
    ap.add_argument("--ext-requests", type=int, default=16,
                    help="requests of the serving measurement in the default line")
    ap.add_argument("--workload", default="blast3d", choices=["blast3d", "radial", "serving", "precision"],
                    help="blast3d: the 384^3 octant case; radial: the batch of 4096 1-D radial blasts; "
                         "serving: a Poisson stream of mixed-size blast cases through the serving loop; "
                         "precision: FP64 against FP32-mode runs of the 384^3 blast and a 512^3 periodic box")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"],
                    help="blast3d and serving: FP64, or the FP32 mode (float intermediates, double state)")
    ap.add_argument("--periodic-n", type=int, default=512, help="precision workload: periodic box grid")
    ap.add_argument("--requests", type=int, default=16, help="serving workload: number of requests")
    ap.add_argument("--nprob", type=int, default=4096, help="radial workload: number of problems")
    args = ap.parse_args()
    if args.workload == "radial" and "--steps" not in sys.argv:
        args.steps = 500            # the radial configuration runs 500 LDDRK4 steps per problem

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if (args.impl == "b200" and torch.cuda.is_available()) else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))

    if args.workload == "radial":
        run_radial(args, rank, world, local, dist)
        if dist is not None:
            dist.destroy_process_group()
        return
    if args.workload == "serving":
        run_serving(args, rank, world, local, dist)
        if dist is not None:
            dist.destroy_process_group()
        return
    if args.workload == "precision":
        run_precision(args, rank, world, local, dist)
        if dist is not None:
            dist.destroy_process_group()
        return

    if args.impl == "reference":
        run_reference(args, rank)
        if dist is not None:
            dist.destroy_process_group()
        return

    from shock_turbulence_b200 import Solver
    from shock_turbulence_b200.replicas import aggregate_rate, max_over_ranks, replica_seed
    torch.cuda.set_device(local)
    fp32 = args.precision == "fp32"
    p = make_params(args.n, device=local, precision=1 if fp32 else 0)
    Q, Y = make_state(p, seed=replica_seed(1, rank))
    s = Solver(p)
    stream = torch.cuda.current_stream()
    s._check(s.lib.st_set_stream(s._h, stream.cuda_stream), "st_set_stream")
    s.set_state(Q, Y)
    s.Compute_gamma(Y)
    s.Compute_hyper(Q, Y)
    t, st = 0.0, 0
    for _ in range(args.warmup):
        t, st = s.step(t, st)
    torch.cuda.synchronize()

    def barrier():
        if dist is not None:
            dist.barrier()

    # ---- device-timed region (inputs resident in HBM) ----
    clocks = ClockSampler(gpu_smi_id(local))
    import ctypes
    c0 = ctypes.c_longlong()
    s.lib.st_launch_count(s._h, ctypes.byref(c0))
    s.lib.st_profile(s._h, 1)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        t, st = s.step(t, st)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    s.lib.st_profile(s._h, 0)
    c1 = ctypes.c_longlong()
    s.lib.st_launch_count(s._h, ctypes.byref(c1))
    buf = ctypes.create_string_buffer(1 << 16)
    s._check(s.lib.st_profile_report(s._h, buf, len(buf)), "st_profile_report")
    prof_sites = json.loads(buf.value.decode())
    # pointwise launches are reported per source site; fold them into one entry
    prof, sites = {}, {}
    for k, v in prof_sites.items():
        key = "k_pointwise" if k.startswith("k_pointwise@") else k
        if key != k:
            sites[k.split("@")[1]] = v
        a = prof.setdefault(key, {"launches": 0, "ms": 0.0, "bytes": 0.0})
        for f in ("launches", "ms", "bytes"):
            a[f] += v[f]
    ms = max_over_ranks(e0.elapsed_time(e1), dist, "cuda")
    cells = args.n ** 3
    value = aggregate_rate(cells, args.steps, ms, world)
    mon = s.monitors()
    finite = bool(math.isfinite(mon[0]) and math.isfinite(mon[5]))
    want_ext = world == 1 and not args.no_extensions and not fp32
    ref_state = s.get_state() if want_ext else None     # FP64 state after warm-up + timed steps

    # ---- end-to-end through the public API with host buffers ----
    import numpy as np
    io_bytes = 6 * cells * 8
    e2e = None
    if args.e2e_steps > 0:
        Qh = torch.from_numpy(np.ascontiguousarray(s.get_state()[0])).pin_memory()
        Yh = torch.from_numpy(np.ascontiguousarray(s.get_state()[1])).pin_memory()
        barrier()
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(args.e2e_steps):
            s.set_state(Qh, Yh)          # H2D of the step's inputs (pinned host)
            t, st = s.step(t, st)
            s.get_state(Qh, Yh)          # D2H of the step's result
        f1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ms_e2e = max_over_ranks(f0.elapsed_time(f1), dist, "cuda")
        e2e = aggregate_rate(cells, args.e2e_steps, ms_e2e, world)

    # ---- roofline of the dominant kernel ----
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peak, peak_src = float(json.load(open(peaks_path))["hbm_gbs"]), "measured"
    else:
        peak, peak_src = 6650.0, "fallback"
    # k_pointwise is a family of distinct kernels (one per source site), so the
    # dominant single kernel is taken among the others
    dom = max((k for k in prof if prof[k]["bytes"] > 0 and k != "k_pointwise"), key=lambda k: prof[k]["ms"])
    d = prof[dom]
    achieved = d["bytes"] / (d["ms"] / 1e3) / 1e9
    step_ms_all = sum(v["ms"] for v in prof.values())
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_src,
                "traffic": (traffic_ratio(dom) * d["bytes"] / d["launches"]) if traffic_ratio(dom) else None,
                "traffic_basis": (f"ncu dram read+write / algorithmic bytes of a 256^3 capture of {dom} "
                                  "(profiles/ncu_traffic.txt) times the algorithmic bytes per launch")
                                 if traffic_ratio(dom) else f"no ncu DRAM capture of {dom}",
                "algorithmic_bytes_per_launch": d["bytes"] / d["launches"],
                "avg_launch_ms": d["ms"] / d["launches"],
                "share_of_kernel_time": d["ms"] / step_ms_all if step_ms_all else None,
                "kernels": {k: {"launches": v["launches"], "ms": round(v["ms"], 3),
                                "GB/s": (v["bytes"] / (v["ms"] / 1e3) / 1e9) if v["bytes"] and v["ms"] else None}
                            for k, v in prof.items()},
                "pointwise_sites_ms": {"st_physics.cu:" + k: round(v["ms"], 2)
                                       for k, v in sorted(sites.items(), key=lambda kv: -kv[1]["ms"])[:12]}}
    # the whole step: algorithmic bytes of every launched kernel over their
    # summed device time (each launch counts its own inputs and outputs once,
    # so fusion is neither rewarded nor punished)
    step_bytes = sum(v["bytes"] for v in prof.values())
    if step_ms_all:
        step_gbs = step_bytes / (step_ms_all / 1e3) / 1e9
        roofline["step"] = {"achieved": step_gbs, "frac": step_gbs / peak,
                            "bytes_per_step": step_bytes / args.steps,
                            "kernel_ms_per_step": step_ms_all / args.steps,
                            "bytes_per_cell_per_stage": step_bytes / args.steps / cells / 10}
    if not fp32:
        # the reference's operator graph (derivative, filter and Gaussian
        # passes and stage updates at their interface bytes; pointwise passes
        # not counted) moved in the measured step time: how near the step is
        # to the bound an ideal fusion of this graph would have
        g_bytes = GRAPH_BYTES_PER_CELL_STAGE * 10 * cells
        g_gbs = g_bytes / (ms / args.steps / 1e3) / 1e9
        roofline["graph"] = {"bytes_per_cell_per_stage": GRAPH_BYTES_PER_CELL_STAGE, "bytes_per_step": g_bytes,
                             "achieved": g_gbs, "frac": g_gbs / peak,
                             "basis": "interface bytes of the reference operator calls of one step (count of the "
                                      "instrumented CPU oracle, tests/test_graph_bytes.py) / ms_per_step"}
    for k, v in prof.items():
        if v["bytes"] and v["ms"]:
            roofline["kernels"][k]["frac"] = round(v["bytes"] / (v["ms"] / 1e3) / 1e9 / peak, 3)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        rate, el = oracle_rate(args.cpu_n, 3, 1, threads)
        cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"CPU oracle, {args.cpu_n}^3 sample of the same workload, 1 warm-up + 3 timed steps "
                         f"({el:.1f} s), {threads} OpenMP threads"}
        cpu["single_core"] = single_core_rate()
        cpu["cpu_model"] = cpu_model()

    ext = None
    if want_ext:
        s.close()
        s = None
        ext = {"fp32_mode": fp32_extension(args, local, Q, Y, ref_state, value),
               "serving": serving_extension(args, local, value)}

    if rank == 0:
        line = {
            "metric": METRIC_FP32 if fp32 else METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 intermediates / f64 state" if fp32 else "f64",
            "data": "synthetic (seeded solenoidal turbulence + Gaussian blast)",
            "config": {"workload": f"blast wave in isotropic turbulence, {args.n}^3 octant, "
                                   f"{'FP32 mode' if fp32 else 'FP64'}, two-species _mf "
                                   "physics (Y=1), Re=100 viscous term on, artificial viscosity on, CFL 0.5",
                       "grid": args.n, "cells": cells, "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (one field is %.0f MB)" % (cells * 8 / 1e6),
                       "finite": finite,
                       # stages per step differ between the families (10 here, 11 for the sf ones)
                       "rk_stages_per_step": 10, "mcell_stages_per_s": value * 10},
            "e2e": ({"value": e2e, "unit": UNIT, "h2d_bytes_per_step": io_bytes, "d2h_bytes_per_step": io_bytes,
                     "steps": args.e2e_steps} if e2e is not None else None),
            "gpu_launches": int(c1.value - c0.value),
            "roofline": roofline,
            "cpu_baseline": cpu,
            "clocks": clk,
        }
        if ext is not None:
            line["extensions"] = ext
        print(json.dumps(line), flush=True)
    if s is not None:
        s.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
