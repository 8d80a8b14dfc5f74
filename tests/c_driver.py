"""Builds the C driver (sparc2_b200/host/sparc_driver.c) and writes its raw
input files for a test case."""
import ctypes as C
import os
import subprocess

import numpy as np

from sparc2_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "sparc2_b200", "host", "sparc_driver.c")
LIBDIR = os.path.join(ROOT, "sparc2_b200", "_lib")


def build(out_dir):
    from sparc2_b200 import build as B
    if not os.path.exists(B.LIB):  # the prebuilt in-tree library otherwise
        B.build()
    exe = os.path.join(str(out_dir), "sparc_driver")
    subprocess.check_call(["gcc", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                           SRC, "-o", exe, "-L", LIBDIR, "-lsparc_gpu",
                           "-Wl,-rpath," + LIBDIR])
    return exe


def write_inputs(d, params, bg, source=None):
    d = str(d)
    with open(os.path.join(d, "params.bin"), "wb") as f:
        f.write(bytes(params))
    if source is not None:
        with open(os.path.join(d, "source.bin"), "wb") as f:
            f.write(C.string_at(C.addressof(source), C.sizeof(source)))
        keep = getattr(source, "_keep", None)
        if source.kind == abi.SPARC_SRC_PSR:
            with open(os.path.join(d, "pulses.bin"), "wb") as f:
                f.write(C.string_at(C.addressof(keep), C.sizeof(keep)))
        elif source.kind == abi.SPARC_SRC_RANDOM:
            np.ascontiguousarray(keep, dtype="<f8").tofile(os.path.join(d, "series.bin"))
    names = ["rho0", "pre0", "cs0", "zaxis", "grav"]
    if params.magnetic == 2:
        names += ["bx0", "by0", "bz0"]
    for n in names:
        np.ascontiguousarray(bg[n], dtype="<f8").tofile(os.path.join(d, n + ".bin"))


def run(exe, d, first, count, *extra):
    return subprocess.run([exe, str(d), str(first), str(count), *extra],
                          capture_output=True, text=True, timeout=600)
