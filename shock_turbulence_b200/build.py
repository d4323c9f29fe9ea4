"""Builds the sm_100a CUDA library ``libst_b200.so`` in-tree with nvcc.

Everything is compiled with ``--fmad=false`` so that every product and sum
rounds as the reference source writes it.  (Contracting the line kernels'
multiply-adds was measured: 1.5-4 % faster operators, but the artificial
viscosity coefficients, which take high-order derivatives of nearly constant
fields, then moved by up to 17 % on a periodic test case against the
oracle.)  Each source compiles to its own object in ``_build/`` (in parallel;
the line-kernel translation units hold most of the template instantiations),
then nvcc links the shared library.
"""
import os
import subprocess
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libst_b200.so")
SOURCES = ["st_kernels.cu", "st_kernels_cyc.cu", "st_kernels_f32.cu", "st_kernels_cyc_f32.cu", "st_physics.cu",
           "st_radial.cu", "st_noalloc.cu", "st_diag.cu", "st_tables.cpp", "st_api.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "--extended-lambda", "-std=c++17", "-Xcompiler", "-fPIC"]


def _newest_source_mtime():
    paths = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    paths.append(os.path.join(HERE, "..", "include", "st_b200.h"))
    paths.append(os.path.abspath(__file__))
    return max(os.path.getmtime(p) for p in paths)


def _compile(src, verbose):
    obj = os.path.join(OBJ, os.path.splitext(src)[0] + ".o")
    cmd = ["nvcc", *NVCC_FLAGS, "--fmad=false", "-c", "-o", obj, os.path.join(CSRC, src)]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    return obj


def build(force=False, verbose=False, jobs=None):
    """Compile the library unless an up-to-date copy exists; returns its path."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _newest_source_mtime():
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    jobs = jobs or min(len(SOURCES), os.cpu_count() or 1)
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    cmd = ["nvcc", *ARCH, "-shared", "-Xlinker", "--no-undefined", "-o", LIB] + objs
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose=True))
