"""Visual output on the CPU: the oracle's MakePaddedArrays against a numpy
statement of src/vis_silo_mf.f:486-686 (primitive variables, clamped
padding, padded coordinates), the file-name rule and the VTK reader on a
file assembled here byte by byte."""
import os

import numpy as np

from shock_turbulence_b200.params import default_params
from shock_turbulence_b200.visual import FIELD_OF, NAMES, read_vtk, visual_path


def test_oracle_padded_arrays(oracle_mod):
    from shock_turbulence_b200.initial import blast_in_turbulence
    p = default_params(16, 32, 24, length=2.0)
    p.z_start = 1.5
    Q, Y = blast_in_turbulence(p, k0=4, mach_t=0.1, p_ratio=20.0, radius_cells=3, seed=4)
    Y = np.ascontiguousarray(np.clip(Y - 0.4 * np.random.default_rng(1).random(Y.shape), 0.0, 1.0))
    o = oracle_mod.Oracle(p)
    o.set_state(Q, Y)
    o.compute_gamma(Y)
    G = np.random.default_rng(3).standard_normal((4,) + o.shape)
    W, xx, yy, zz = o.make_padded_arrays(G)
    gam = o.get_common("gamma_eff")
    ix = np.arange(p.nx + 1).clip(max=p.nx - 1)
    kz = np.arange(p.nz + 1).clip(max=p.nz - 1)
    jy = np.arange(p.ny + 1).clip(max=p.ny - 1)

    def pad(a):
        return a[np.ix_(ix, kz, jy)]

    q1, q2, q3, q4, q5 = Q
    vs = 1.0 / q4
    P = (gam - 1.0) * (q5 - 0.5 * vs * (q1 * q1 + q2 * q2 + q3 * q3))
    want = [q1 / q4, q2 / q4, q3 / q4, q4, P, G[0], G[1], G[2], G[3], gam, Y]
    for f in range(11):
        assert np.array_equal(W[f], pad(want[f])), f
    for cor, n, s0, ln in ((xx, p.nx, p.x_start, p.x_leng), (yy, p.ny, p.y_start, p.y_leng),
                           (zz, p.nz, p.z_start, p.z_leng)):
        g = s0 + ln * np.arange(n) / (n - 1)
        assert np.array_equal(cor[:n], g) and cor[n] == g[-1] + (g[1] - g[0])


def test_visual_path_rule():
    assert visual_path("vis", "srm", 7) == os.path.join("vis", "007", "srm.000.vtk")
    assert visual_path("/a/b", "p", 123) == os.path.join("/a/b", "123", "p.000.vtk")


def test_reader_on_an_assembled_file(tmp_path):
    ny, nz, nx = 3, 2, 4
    rng = np.random.default_rng(0)
    cy, cz, cx = rng.random(ny), rng.random(nz), rng.random(nx)
    fields = {n: rng.standard_normal((nx, nz, ny)) for n in NAMES}
    b = bytearray(b"# vtk DataFile Version 3.0\ntitle\nBINARY\nDATASET RECTILINEAR_GRID\n")
    b += b"FIELD FieldData 2\nTIME 1 1 double\n" + np.array([0.75], ">f8").tobytes() + b"\n"
    b += b"CYCLE 1 1 int\n" + np.array([42], ">i4").tobytes() + b"\n"
    b += b"DIMENSIONS %d %d %d\n" % (ny, nz, nx)
    for ax, c in (("X", cy), ("Y", cz), ("Z", cx)):
        b += b"%s_COORDINATES %d double\n" % (ax.encode(), c.size) + c.astype(">f8").tobytes() + b"\n"
    b += b"POINT_DATA %d\n" % (nx * ny * nz)
    for n in NAMES:
        b += b"SCALARS %s double 1\nLOOKUP_TABLE default\n" % n.encode() + fields[n].astype(">f8").tobytes() + b"\n"
    path = tmp_path / "f.vtk"
    path.write_bytes(bytes(b))
    v = read_vtk(str(path))
    assert v["time"] == 0.75 and v["cycle"] == 42 and v["dims"] == (ny, nz, nx)
    assert np.array_equal(v["coords"]["y"], cy) and np.array_equal(v["coords"]["x"], cx)
    for n in NAMES:
        assert np.array_equal(v["fields"][n], fields[n])
    assert sorted(FIELD_OF.values()) == list(range(11))
