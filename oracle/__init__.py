"""TEST INFRASTRUCTURE: ctypes wrapper of the oracle (sparc_oracle.cpp).

The oracle is a CPU FP64 restatement of the reference time step.  Only the
tests, __graft_entry__.smoke() and bench.py's CPU baseline / reference arm
use it, as the checker or the timed CPU baseline; the product library never
loads it.  Parity is unpinned by reference tests (the reference has none and
cannot be built here); see oracle/sparc_oracle.h.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from sparc2_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "sparc_oracle.cpp")
BUILD_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD_DIR, "libsparc_oracle.so")

CXXFLAGS = ["-std=c++17", "-O3", "-march=x86-64-v3", "-ffp-contract=off",
            "-fopenmp", "-fPIC", "-shared"]


def build(force=False):
    """Compile the oracle with g++ into oracle/_build (git-ignored)."""
    os.makedirs(BUILD_DIR, exist_ok=True)
    deps = [SRC, os.path.join(HERE, "sparc_oracle.h"),
            os.path.join(HERE, "..", "include", "sparc_gpu.h")]
    if (not force and os.path.exists(LIB) and
            os.path.getmtime(LIB) >= max(os.path.getmtime(d) for d in deps)):
        return LIB
    tmp = LIB + ".tmp"
    subprocess.check_call(["g++", *CXXFLAGS, "-o", tmp, SRC])
    os.replace(tmp, LIB)
    return LIB


_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        lib = C.CDLL(LIB)
        d = C.POINTER(C.c_double)
        h = C.c_void_p
        lib.orc_create.restype = h
        lib.orc_create.argtypes = [C.POINTER(abi.SparcParams), d, d, d, d, d,
                                   d, d, d, C.c_char_p, C.c_int]
        lib.orc_destroy.argtypes = [h]
        lib.orc_set_source.argtypes = [h, C.POINTER(abi.SparcSource)]
        lib.orc_sizes.argtypes = [h, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        lib.orc_set_state.argtypes = [h, d, d]
        lib.orc_get_state.argtypes = [h, d, d]
        lib.orc_step.argtypes = [h, C.c_int64]
        lib.orc_filter_vars.argtypes = [h, C.c_int64]
        lib.orc_run.argtypes = [h, C.c_int64, C.c_int64]
        lib.orc_diagnostics.argtypes = [h, C.POINTER(abi.SparcDiag)]
        lib.orc_derivative.argtypes = [h, C.c_int, C.c_int, d, d]
        lib.orc_filter_field.argtypes = [h, C.c_int, d, d]
        lib.orc_get_coeff.argtypes = [h, C.c_char_p, d, C.POINTER(C.c_int64)]
        lib.orc_get_scalars.argtypes = [h, d]
        lib.orc_forcing.argtypes = [h, C.c_int64, d]
        lib.orc_rhs.argtypes = [h, C.c_int64, d, d, d, d]
        lib.orc_set_threads.argtypes = [C.c_int]
        lib.orc_get_threads.restype = C.c_int
        _lib = lib
    return _lib


def set_threads(n):
    _load().orc_set_threads(int(n))


def get_threads():
    return _load().orc_get_threads()


class Oracle:
    """One simulation on the CPU oracle; mirrors sparc2_b200.Simulation."""

    def __init__(self, params, bg, source=None):
        lib = _load()
        self.lib = lib
        self.params = params
        self.nx, self.ny, self.nz = params.nx, params.ny, params.nz
        self.V = 8 if params.magnetic == 2 else 5
        err = C.create_string_buffer(256)
        f = abi.dptr
        self.h = lib.orc_create(C.byref(params), f(bg["rho0"]), f(bg["pre0"]),
                                f(bg["cs0"]), f(bg.get("bx0")),
                                f(bg.get("by0")), f(bg.get("bz0")),
                                f(np.ascontiguousarray(bg["zaxis"])),
                                f(np.ascontiguousarray(bg["grav"])), err, 256)
        if not self.h:
            raise abi.SparcError(abi.SPARC_ERR_INVALID, "orc_create",
                                 err.value.decode())
        ns, npsi = C.c_int64(), C.c_int64()
        lib.orc_sizes(self.h, C.byref(ns), C.byref(npsi))
        self.n_state, self.n_psi = ns.value, npsi.value
        if source is not None:
            self.set_source(source)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    @property
    def shape(self):
        return (self.nz, self.ny, self.nx)

    def set_source(self, src):
        r = self.lib.orc_set_source(self.h, C.byref(src))
        if r != 0:
            raise abi.SparcError(r, "orc_set_source")

    def set_state(self, a, psi=None):
        a = np.ascontiguousarray(a, dtype=np.float64)
        p = None if psi is None else np.ascontiguousarray(psi, dtype=np.float64)
        self.lib.orc_set_state(self.h, abi.dptr(a), abi.dptr(p))

    def get_state(self):
        a = np.empty((self.V,) + self.shape)
        psi = np.empty(self.n_psi)
        self.lib.orc_get_state(self.h, abi.dptr(a), abi.dptr(psi))
        return a, psi

    def step(self, nn):
        self.lib.orc_step(self.h, int(nn))

    def filter_vars(self, nn):
        self.lib.orc_filter_vars(self.h, int(nn))

    def run(self, first, count):
        return self.lib.orc_run(self.h, int(first), int(count))

    def diagnostics(self):
        d = abi.SparcDiag()
        r = self.lib.orc_diagnostics(self.h, C.byref(d))
        return d, r

    def derivative(self, dir, bc, field):
        field = np.ascontiguousarray(field, dtype=np.float64)
        out = np.empty_like(field)
        r = self.lib.orc_derivative(self.h, dir, bc, abi.dptr(field),
                                    abi.dptr(out))
        if r:
            raise abi.SparcError(r, "orc_derivative")
        return out

    def filter_field(self, dir, field):
        field = np.ascontiguousarray(field, dtype=np.float64)
        out = np.empty_like(field)
        self.lib.orc_filter_field(self.h, dir, abi.dptr(field), abi.dptr(out))
        return out

    def coeff(self, name):
        n = C.c_int64()
        r = self.lib.orc_get_coeff(self.h, name.encode(), None, C.byref(n))
        if r:
            raise abi.SparcError(r, "orc_get_coeff", name)
        out = np.empty(n.value)
        self.lib.orc_get_coeff(self.h, name.encode(), abi.dptr(out),
                               C.byref(n))
        return out

    def scalars(self):
        out = np.empty(12)
        self.lib.orc_get_scalars(self.h, abi.dptr(out))
        keys = ["dimc", "dimrho", "diml", "dimb", "deltat", "stretchx",
                "stretchy", "beta1", "beta2", "beta3", "beta4", "beta5"]
        return dict(zip(keys, out))

    def forcing(self, nn):
        out = np.empty(self.shape)
        self.lib.orc_forcing(self.h, int(nn), abi.dptr(out))
        return out

    def rhs(self, nn, temp, psi=None):
        temp = np.ascontiguousarray(temp, dtype=np.float64)
        scr = np.empty_like(temp)
        spsi = np.empty(self.n_psi)
        p = None if psi is None else np.ascontiguousarray(psi, dtype=np.float64)
        self.lib.orc_rhs(self.h, int(nn), abi.dptr(temp), abi.dptr(p),
                         abi.dptr(scr), abi.dptr(spsi))
        return scr, spsi
