"""Per-operator timing and profiling driver.

Runs one line operator (or the full step) on device-resident fields of an
n^3 grid through the C ABI and prints achieved GB/s of its algorithmic bytes
(every input and output field touched once) from CUDA events on the context
stream.  Used for ncu captures and roofline checks:

    python -m shock_turbulence_b200.opbench --op dfd --n 256 --reps 3
"""
import argparse
import ctypes
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

# op -> (bytes per cell, runner)
OPS = ("dfd", "dfd_add", "d2fd2", "filter", "gauss", "step")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--op", default="dfd", choices=OPS)
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--dirs", default="xyz")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"],
                    help="step: FP64, or the FP32 mode (its line kernels run only inside the step)")
    args = ap.parse_args()

    import torch
    from shock_turbulence_b200 import Solver, default_params
    p = default_params(args.n, re=100.0, precision=1 if args.precision == "fp32" else 0)
    s = Solver(p)
    stream = torch.cuda.current_stream()
    s._check(s.lib.st_set_stream(s._h, stream.cuda_stream), "st_set_stream")
    shape = s.shape
    g = torch.Generator(device="cuda").manual_seed(0)
    F = torch.randn(shape, dtype=torch.float64, device="cuda", generator=g)
    O1 = torch.zeros_like(F)
    O2 = torch.zeros_like(F)
    n3 = args.n ** 3

    if args.op == "step":
        from shock_turbulence_b200.initial import blast_in_turbulence
        Q, Y = blast_in_turbulence(p, k0=8.0, mach_t=0.1, p_ratio=100.0, radius_cells=4.0, seed=1)
        s.set_state(Q, Y)
        s.Compute_gamma(Y)
        s.Compute_hyper(Q, Y)
        state = {"t": 0.0, "s": 0}

        def run(_d):
            state["t"], state["s"] = s.step(state["t"], state["s"])
        bytes_per = 0
    else:
        names = {"dfd": "DFD{}_sym", "dfd_add": "DFD{}_sym", "d2fd2": "D2FD{}2_sym",
                 "filter": "Compact_Filter_{}_sym", "gauss": "Gaussian_Filter_{}"}
        bytes_per = {"dfd": 16, "dfd_add": 24, "d2fd2": 24, "filter": 16, "gauss": 16}[args.op]

        def run(d):
            fn = getattr(s, names[args.op].format(d.upper()))
            if args.op == "dfd":
                fn(F, O1, 0, 1.0)
            elif args.op == "dfd_add":
                fn(F, O1, 1, 1.0)
            elif args.op == "d2fd2":
                fn(F, O1, O2, 1)
            else:
                fn(F, O1)

    out = {}
    for d in (args.dirs if args.op != "step" else "x"):
        for _ in range(args.warmup):
            run(d)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.reps):
            run(d)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.reps
        out[d] = {"ms": ms, "GB/s": (bytes_per * n3 / (ms / 1e3) / 1e9) if bytes_per else None}
    cnt = ctypes.c_longlong()
    s.lib.st_launch_count(s._h, ctypes.byref(cnt))
    print(json.dumps({"op": args.op, "n": args.n, "reps": args.reps, "results": out, "launches": cnt.value}))


if __name__ == "__main__":
    main()
