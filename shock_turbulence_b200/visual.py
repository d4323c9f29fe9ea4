"""Visual files: path rule and reader of the legacy VTK file that
``st_write_visual`` (Write_Visual_Silo, src/vis_silo_mf.f:7-277) writes.

The reference writes a Silo quad mesh (collinear axes "yc", "zc", "xc" of
sizes My+1, Mz+1, Mx+1) with eleven node-centred double variables and the
cycle and time as options.  The Silo library is not part of this build, so
the same content is one binary (big-endian) legacy VTK rectilinear-grid file
(VisIt and ParaView read it): the VTK x axis is the reference's first mesh
axis (y), then z, then x; FIELD data TIME and CYCLE carry the time and step.
"""
import os

import numpy as np

NAMES = ("rho", "U", "V", "W", "P", "omx", "omy", "omz", "dil", "gamma", "Y")
# index into the W(..., 11) fields of MakePaddedArrays of each written name
FIELD_OF = {"rho": 3, "U": 0, "V": 1, "W": 2, "P": 4, "omx": 5, "omy": 6, "omz": 7, "dil": 8, "gamma": 9, "Y": 10}


def visual_path(vis_path, prefix, cue_vis):
    """<vis_path>/<ddd>/<prefix>.000.vtk, ddd the three digits of cue_vis:
    the directory make_dir_ creates (src/dirs.c) and the file name of group
    0 (src/vis_silo_mf.f:97-106)."""
    c = int(cue_vis)
    d = f"{(c // 100) % 10}{(c % 100) // 10}{c % 10}"
    return os.path.join(os.fsdecode(vis_path), d, f"{os.fsdecode(prefix)}.000.vtk")


def read_vtk(path):
    """Read a file of ``st_write_visual``: returns a dict with 'time',
    'cycle', 'dims' (My+1, Mz+1, Mx+1), 'coords' {'y','z','x'} and 'fields'
    {name: array of shape (Mx+1, Mz+1, My+1)}."""
    data = open(path, "rb").read()
    pos = 0

    def line():
        nonlocal pos
        e = data.index(b"\n", pos)
        s = data[pos:e].decode("ascii")
        pos = e + 1
        return s

    def block(n, dt):
        nonlocal pos
        a = np.frombuffer(data, dtype=dt, count=n, offset=pos).astype(dt.newbyteorder("="))
        pos += n * dt.itemsize
        if data[pos:pos + 1] == b"\n":
            pos += 1
        return a

    if not line().startswith("# vtk DataFile"):
        raise ValueError(f"{path}: not a legacy VTK file")
    out = {"title": line(), "fields": {}, "coords": {}}
    if line().strip() != "BINARY":
        raise ValueError(f"{path}: not a binary VTK file")
    if line().strip() != "DATASET RECTILINEAR_GRID":
        raise ValueError(f"{path}: not a rectilinear grid")
    f8, i4 = np.dtype(">f8"), np.dtype(">i4")
    axes = {"X": "y", "Y": "z", "Z": "x"}
    while pos < len(data):
        words = line().split()
        if not words:
            continue
        key = words[0]
        if key == "FIELD":
            for _ in range(int(words[2])):
                name, _, n, typ = line().split()
                v = block(int(n), f8 if typ == "double" else i4)
                out["time" if name == "TIME" else "cycle"] = float(v[0]) if typ == "double" else int(v[0])
        elif key == "DIMENSIONS":
            out["dims"] = tuple(int(w) for w in words[1:4])
        elif key.endswith("_COORDINATES"):
            out["coords"][axes[key[0]]] = block(int(words[1]), f8)
        elif key == "POINT_DATA":
            npts = int(words[1])
        elif key == "SCALARS":
            line()                                   # LOOKUP_TABLE default
            ny1, nz1, nx1 = out["dims"]
            out["fields"][words[1]] = block(npts, f8).reshape(nx1, nz1, ny1)
        else:
            raise ValueError(f"{path}: unexpected keyword {key}")
    return out
