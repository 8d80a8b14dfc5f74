"""Builds libsparc_gpu.so in-tree for sm_100a with nvcc.

The setup translation unit is compiled with -fmad=false so the FP64
coefficient arrays are a plain IEEE evaluation of the reference's
expressions; the time-step kernels keep FMA contraction.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libsparc_gpu.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "--extended-lambda",
          "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall"]
UNITS = {
    "setup.cu": ["-fmad=false"],
    "step.cu": [],
    "step32.cu": [],
    "api.cu": [],
    "batch.cu": [],
    "noalloc.cu": [],
    "serve.cu": [],
    "damping.cu": [],
}
HEADERS = ["internal.h", "mhd_body.cuh", "random_forcing.cuh", "filter_body.cuh",
           "tmem_window.cuh", "tma_util.cuh"]
# host C units (gcc): the .trol reader
HOST_UNITS = {"sparc_trol.c": ["-O2", "-std=c99", "-Wall", "-fPIC"]}
HOST = os.path.join(HERE, "host")


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or c == "nvcc"):
            return c
    return "nvcc"


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, ptxas_v=False):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS]
    hdrs.append(os.path.join(HERE, "..", "include", "sparc_gpu.h"))
    objs = []
    for unit, flags in HOST_UNITS.items():
        src = os.path.join(HOST, unit)
        obj = os.path.join(BUILD, unit + ".o")
        objs.append(obj)
        deps = [src, os.path.join(HERE, "..", "include", "sparc_trol.h"), hdrs[-1], __file__]
        if force or _stale(obj, deps):
            cmd = ["gcc", *flags, "-I", os.path.join(HERE, "..", "include"), "-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.check_call(cmd)
    for unit, extra in UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(BUILD, unit + ".o")
        objs.append(obj)
        if force or _stale(obj, [src, *hdrs, __file__]):
            cmd = [nvcc(), *ARCH, *COMMON, *extra, "-c", src, "-o", obj]
            if ptxas_v:
                cmd.insert(1, "-Xptxas=-v")
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.check_call(cmd)
    if force or _stale(LIB, objs):
        tmp = LIB + ".tmp"
        subprocess.check_call([nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-lcufft"])
        _check_resolved(tmp)
        os.replace(tmp, LIB)
    return LIB


def _check_resolved(lib):
    """A shared library links with unresolved symbols; refuse one that
    leaves any of its own (namespace sparc) undefined."""
    out = subprocess.run(["nm", "-u", "-C", lib], capture_output=True, text=True)
    if out.returncode != 0:
        return  # no nm: nothing to check with
    missing = [l.strip() for l in out.stdout.splitlines() if "sparc::" in l]
    if missing:
        os.remove(lib)
        raise RuntimeError("unresolved library symbols: " + "; ".join(missing))


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          ptxas_v="--ptxas" in sys.argv)
