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


def trol_text(params, source=None, solartime_h=None):
    """A .trol control file (the reference's key = value format) holding
    params and the source's .trol keys, written in an order that respects
    the reader's order-sensitive keys (USE_PML/USE_HPML before PERIODIC and
    the PML lines, PULSE before pulse_*, timestep before t_xy/t_z)."""
    p = params
    L = [f"nx = {p.nx}", f"ny = {p.ny}", f"nz = {p.nz}",
         f"xlength = {p.xlength!r}", f"ylength = {p.ylength!r}",
         f"timestep = {p.timestep!r}",
         f"STABILISE = {p.stabilise}", "DAMPING = 0", "MODE = 0", "FLOWS = 0",
         "TWOD = 0", f"MAGNETIC = {p.magnetic}", f"maxva = {p.maxva!r}",
         f"block_x = {p.block_x}", f"block_y = {p.block_y}", f"block_z = {p.block_z}",
         f"USE_PML = {p.use_pml}", f"USE_HPML = {p.use_hpml}",
         f"PERIODIC = {p.periodic}"]
    for key, n, arr in (("xpmlb", p.npml_xb, p.pml_xb), ("xpmlt", p.npml_xt, p.pml_xt),
                        ("ypmlb", p.npml_yb, p.pml_yb), ("ypmlt", p.npml_yt, p.pml_yt),
                        ("zpmlb", p.npml_zb, p.pml_zb), ("zpmlt", p.npml_zt, p.pml_zt)):
        L.append(f"{key} = {n}," + ",".join(repr(float(v)) for v in arr))
    L += [f"sp_str = {p.sp_str!r}", f"sp_length = {p.sp_length!r}",
          f"sp_decay = {p.sp_decay!r}",
          f"filter_mode_xy = {p.filter_mode_xy}", f"filter_mode_z = {p.filter_mode_z}",
          f"s_xy = {p.s_xy!r}", f"s_z = {p.s_z!r}", f"t_xy = {p.t_xy!r}", f"t_z = {p.t_z!r}"]
    if source is not None:
        kind = {abi.SPARC_SRC_PULSE: 1, abi.SPARC_SRC_PSR: 2, abi.SPARC_SRC_RANDOM: 0}[source.kind]
        L.append(f"PULSE = {kind}")
        L.append(f"pulse_dir = {source.dir}")
        if kind == 1:
            for k in ("t0", "t1", "st", "px", "py", "pz", "sr", "sz", "amp"):
                L.append(f"pulse_{k} = {getattr(source, k)!r}")
    if solartime_h is not None:
        L.append(f"solartime = {solartime_h!r}")
    L.append('simname = "test run"')
    return "\n".join(L) + "\n"
