"""Python host side of libsparc_gpu.so: one SPARC simulation on one GPU.

Mirrors the reference driver's calls on the hot path -- STEP
(step.f90:20), FILTER_VARS (derivatives.f90:659) and the per-iteration
diagnostics (driver.f90:161-183) -- through the C ABI of
include/sparc_gpu.h.  There is no CPU fallback: constructing a Simulation
without the built library or without an sm_100 GPU raises.
"""
import ctypes as C

import numpy as np

from . import abi


class Simulation:
    """A handle on the device state of one simulation.

    params: abi.SparcParams; bg: dict with rho0, pre0, cs0 (and bx0, by0,
    bz0 for MHD) as (nz, ny, nx) float64 arrays in cgs units, zaxis (Mm) and
    grav (cm/s^2); source: abi.SparcSource or None.
    """

    def __init__(self, params, bg, source=None, device=0):
        self.lib = abi.load()
        self.params = params
        self.nx, self.ny, self.nz = params.nx, params.ny, params.nz
        self.V = 8 if params.magnetic == 2 else 5
        h = C.c_void_p()
        r = self.lib.sparc_create(C.byref(params), int(device), C.byref(h))
        if r != abi.SPARC_OK:
            raise abi.SparcError(r, "sparc_create",
                                 self.lib.sparc_last_error(None).decode())
        self.h = h
        f = abi.dptr

        def arr(key):
            v = bg.get(key)
            return None if v is None else np.ascontiguousarray(v, dtype=np.float64)

        self._check(self.lib.sparc_set_background(
            self.h, f(arr("rho0")), f(arr("pre0")), f(arr("cs0")),
            f(arr("bx0")), f(arr("by0")), f(arr("bz0")), f(arr("zaxis")),
            f(arr("grav"))), "sparc_set_background")
        ns, npsi = C.c_int64(), C.c_int64()
        self.lib.sparc_sizes(self.h, C.byref(ns), C.byref(npsi))
        self.n_state, self.n_psi = ns.value, npsi.value
        self._source = None
        if source is not None:
            self.set_source(source)

    # -------------------------------------------------------------- helpers
    def _check(self, r, where):
        if r != abi.SPARC_OK:
            raise abi.SparcError(r, where,
                                 self.lib.sparc_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.sparc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def shape(self):
        return (self.nz, self.ny, self.nx)

    # ---------------------------------------------------------------- state
    def set_source(self, src):
        self._source = src            # the pulse table must outlive the call
        self._check(self.lib.sparc_set_source(self.h, C.byref(src)),
                    "sparc_set_source")

    def set_state(self, a, psi=None):
        a = np.ascontiguousarray(a, dtype=np.float64)
        assert a.size == self.n_state
        p = None if psi is None else np.ascontiguousarray(psi, dtype=np.float64)
        self._check(self.lib.sparc_set_state(self.h, abi.dptr(a), abi.dptr(p)),
                    "sparc_set_state")

    def get_state(self):
        a = np.empty((self.V,) + self.shape)
        psi = np.empty(self.n_psi)
        self._check(self.lib.sparc_get_state(self.h, abi.dptr(a), abi.dptr(psi)),
                    "sparc_get_state")
        return a, psi

    # ------------------------------------------------------------ time step
    def step(self, nn):
        """STEP of driver iteration nn (asynchronous)."""
        self._check(self.lib.sparc_step(self.h, int(nn)), "sparc_step")

    def filter_vars(self, nn):
        """FILTER_VARS after iteration nn (asynchronous)."""
        self._check(self.lib.sparc_filter_vars(self.h, int(nn)),
                    "sparc_filter_vars")

    def run(self, first, count):
        """Driver iterations first..first+count-1 as CUDA graphs."""
        self._check(self.lib.sparc_run(self.h, int(first), int(count)),
                    "sparc_run")

    @property
    def zchunk(self):
        """z extent of the stage kernels' work items (layers)."""
        z = C.c_int()
        self._check(self.lib.sparc_get_zchunk(self.h, C.byref(z)), "sparc_get_zchunk")
        return z.value

    def set_zchunk(self, zchunk):
        self._check(self.lib.sparc_set_zchunk(self.h, int(zchunk)), "sparc_set_zchunk")

    def tune(self, first, steps_per_trial=2):
        """Runs the z-extent autotuner from iteration `first` (real driver
        iterations, as sparc_run); returns (next iteration, extent)."""
        nxt, best = C.c_int64(), C.c_int()
        self._check(self.lib.sparc_tune(self.h, int(first), int(steps_per_trial),
                                        C.byref(nxt), C.byref(best)), "sparc_tune")
        return nxt.value, best.value

    def diagnostics(self):
        """(sparc_diag, status): status is SPARC_ERR_UNSTABLE after a
        failed iteration, SPARC_OK otherwise."""
        d = abi.SparcDiag()
        r = self.lib.sparc_diagnostics(self.h, C.byref(d))
        if r not in (abi.SPARC_OK, abi.SPARC_ERR_UNSTABLE):
            self._check(r, "sparc_diagnostics")
        return d, r

    def synchronize(self):
        self._check(self.lib.sparc_synchronize(self.h), "sparc_synchronize")

    @property
    def stream(self):
        s = C.c_void_p()
        self._check(self.lib.sparc_stream(self.h, C.byref(s)), "sparc_stream")
        return s.value or 0

    @property
    def launch_count(self):
        n = C.c_int64()
        self._check(self.lib.sparc_launch_count(self.h, C.byref(n)),
                    "sparc_launch_count")
        return n.value

    # ------------------------------------------------------- unit entries
    def derivative(self, dir, bc, field):
        field = np.ascontiguousarray(field, dtype=np.float64)
        out = np.empty_like(field)
        self._check(self.lib.sparc_derivative(self.h, dir, bc, abi.dptr(field),
                                              abi.dptr(out)), "sparc_derivative")
        return out

    def filter_field(self, dir, field):
        field = np.ascontiguousarray(field, dtype=np.float64)
        out = np.empty_like(field)
        self._check(self.lib.sparc_filter_field(self.h, dir, abi.dptr(field),
                                                abi.dptr(out)),
                    "sparc_filter_field")
        return out

    def coeff(self, name):
        n = C.c_int64()
        self._check(self.lib.sparc_get_coeff(self.h, name.encode(), None,
                                             C.byref(n)), "sparc_get_coeff")
        out = np.empty(n.value)
        self._check(self.lib.sparc_get_coeff(self.h, name.encode(),
                                             abi.dptr(out), C.byref(n)),
                    "sparc_get_coeff")
        return out

    def scalars(self):
        out = np.empty(12)
        self._check(self.lib.sparc_get_scalars(self.h, abi.dptr(out)),
                    "sparc_get_scalars")
        keys = ["dimc", "dimrho", "diml", "dimb", "deltat", "stretchx",
                "stretchy", "beta1", "beta2", "beta3", "beta4", "beta5"]
        return dict(zip(keys, out))
