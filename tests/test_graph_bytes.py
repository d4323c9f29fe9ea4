"""The reference operator graph's interface bytes per cell and RK stage,
counted by the instrumented CPU oracle over one main-loop step of the _mf
blast (src/main_mf.f:137-143 with the Re > 0 viscous terms and the
artificial viscosity on), equal the figure bench.py reports its step
against (roofline.graph)."""
import numpy as np

import bench
from shock_turbulence_b200.params import default_params


def test_graph_bytes_per_cell_and_stage(oracle_mod):
    from shock_turbulence_b200.initial import blast_in_turbulence
    for grid in ((32, 32, 32), (16, 32, 48)):
        p = default_params(*grid, re=100.0, c_beta_scale=1.75)
        Q, Y = blast_in_turbulence(p, k0=4, mach_t=0.1, p_ratio=100.0, radius_cells=3, seed=1)
        o = oracle_mod.Oracle(p)
        o.set_state(Q, Y)
        o.compute_gamma(Y)
        o.compute_hyper(Q, Y)
        oracle_mod.graph_bytes(reset=True)
        o.step(0.0, 0)
        per = oracle_mod.graph_bytes(reset=True) / np.prod(grid) / 10
        assert per == bench.GRAPH_BYTES_PER_CELL_STAGE, (grid, per)
