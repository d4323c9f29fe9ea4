"""Visual output (src/vis_silo_mf.f) on the GPU against the oracle:
MakePaddedArrays (the eleven node fields of the padded grid and its
coordinates) and Write_Visual_Silo's file, read back."""
import os

import numpy as np
import pytest

from shock_turbulence_b200.params import default_params
from shock_turbulence_b200.visual import FIELD_OF, NAMES, read_vtk

pytestmark = pytest.mark.gpu
GRID = (48, 32, 64)            # (nx, ny, nz)


@pytest.fixture(scope="module")
def pair(oracle_mod):
    from shock_turbulence_b200 import Solver
    from shock_turbulence_b200.initial import blast_in_turbulence
    p = default_params(*GRID, length=2.0, re=100.0)
    p.x_start, p.y_start, p.z_start = 0.25, -0.5, 0.0
    Q, Y = blast_in_turbulence(p, k0=4, mach_t=0.1, p_ratio=20.0, radius_cells=4, seed=11)
    Y = np.ascontiguousarray(np.clip(Y - 0.3 * np.random.default_rng(2).random(Y.shape), 0.0, 1.0))
    s, o = Solver(p), oracle_mod.Oracle(p)
    for h in (s, o):
        h.set_state(Q, Y)
    s.Compute_gamma(Y)
    o.compute_gamma(Y)
    yield s, o
    s.close()


def test_padded_arrays_match_the_oracle(pair):
    """Same state, gamma_eff and Grad in, bit-identical fields out (the
    primitive variables take one division or product chain per value)."""
    s, o = pair
    G, _, _ = s.Compute_Grad()
    W, xx, yy, zz = s.MakePaddedArrays(G)
    Wo, xo, yo, zo = o.make_padded_arrays(G)
    assert W.shape == (11, GRID[0] + 1, GRID[2] + 1, GRID[1] + 1)
    for f in range(11):
        assert np.array_equal(W[f], Wo[f]), f
    for a, b in ((xx, xo), (yy, yo), (zz, zo)):
        assert np.array_equal(a, b)
    assert xx[0] == 0.25 and yy[0] == -0.5
    # the padding repeats the last node of each direction
    assert np.array_equal(W[:, -1], W[:, -2]) and np.array_equal(W[:, :, -1], W[:, :, -2])
    assert np.array_equal(W[:, :, :, -1], W[:, :, :, -2])


def test_grad_is_computed_when_not_given(pair):
    s, _ = pair
    G, _, _ = s.Compute_Grad()
    W1, *_ = s.MakePaddedArrays(G)
    W2, *_ = s.MakePaddedArrays(None)
    assert np.array_equal(W1, W2)


def test_visual_file_round_trip(pair, tmp_path):
    s, _ = pair
    W, xx, yy, zz = s.MakePaddedArrays()
    path = s.Write_Visual_Silo(1.25, 7, str(tmp_path), "srm", 12)
    assert path == os.path.join(str(tmp_path), "012", "srm.000.vtk") and os.path.exists(path)
    v = read_vtk(path)
    assert v["time"] == 1.25 and v["cycle"] == 7
    assert v["dims"] == (GRID[1] + 1, GRID[2] + 1, GRID[0] + 1)
    assert np.array_equal(v["coords"]["x"], xx) and np.array_equal(v["coords"]["y"], yy)
    assert np.array_equal(v["coords"]["z"], zz)
    assert list(v["fields"]) == list(NAMES)
    for name in NAMES:
        assert np.array_equal(v["fields"][name], W[FIELD_OF[name]]), name
    # a second file of the same cue replaces the first
    s.Write_Visual_Silo(2.5, 8, str(tmp_path), "srm", 12)
    assert read_vtk(path)["cycle"] == 8


def test_bad_arguments_are_refused(pair, tmp_path):
    from shock_turbulence_b200.api import StError
    s, _ = pair
    with pytest.raises(StError):
        s.Write_Visual_Silo(0.0, 0, str(tmp_path), "srm", 1000)
    with pytest.raises(StError):
        s.Write_Visual_Silo(0.0, 0, str(tmp_path / "missing" / "deeper"), "srm", 1)
