"""Python host side of the batched engine (sparc_batch_* of
include/sparc_gpu.h): many SPARC_FP32 simulations advanced together, one
persistent launch per RK stage over a device (simulation, tile, z-chunk)
work-list, each step one CUDA-graph launch.

The reference has no counterpart (one simulation per MPI job); the member
simulations are ordinary `Simulation` handles and keep their state when
they leave the batch.
"""
import ctypes as C

import numpy as np

from . import abi


class Batch:
    def __init__(self, capacity, device=0):
        self.lib = abi.load()
        self.capacity = int(capacity)
        b = C.c_void_p()
        r = self.lib.sparc_batch_create(int(device), self.capacity, C.byref(b))
        if r != abi.SPARC_OK:
            raise abi.SparcError(r, "sparc_batch_create", "")
        self.b = b
        self.members = {}

    def _check(self, r, where):
        if r != abi.SPARC_OK:
            raise abi.SparcError(r, where,
                                 self.lib.sparc_batch_last_error(self.b).decode())

    def close(self):
        if getattr(self, "b", None):
            self.lib.sparc_batch_destroy(self.b)
            self.b = None
            self.members = {}

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def add(self, sim, first, count):
        """Adds a Simulation (SPARC_FP32) that will run driver iterations
        first .. first+count-1; returns its slot."""
        slot = C.c_int()
        self._check(self.lib.sparc_batch_add(self.b, sim.h, int(first),
                                             int(count), C.byref(slot)),
                    "sparc_batch_add")
        self.members[slot.value] = sim
        return slot.value

    def remove(self, slot):
        self._check(self.lib.sparc_batch_remove(self.b, int(slot)),
                    "sparc_batch_remove")
        return self.members.pop(slot)

    def run(self, steps):
        self._check(self.lib.sparc_batch_run(self.b, int(steps)),
                    "sparc_batch_run")

    def remaining(self):
        out = np.zeros(self.capacity, dtype=np.int64)
        self._check(self.lib.sparc_batch_remaining(
            self.b, out.ctypes.data_as(C.POINTER(C.c_int64))),
            "sparc_batch_remaining")
        return out

    def set_tiles(self, zchunk_mhd, zchunk_quiet):
        self._check(self.lib.sparc_batch_set_tiles(self.b, int(zchunk_mhd),
                                                   int(zchunk_quiet)),
                    "sparc_batch_set_tiles")

    def tiles(self):
        m, q = C.c_int(), C.c_int()
        self._check(self.lib.sparc_batch_get_tiles(self.b, C.byref(m),
                                                   C.byref(q)),
                    "sparc_batch_get_tiles")
        return m.value, q.value

    def tune(self, steps_per_trial=2):
        """Runs the autotuner (real steps of the members); returns the
        chosen (zchunk_mhd, zchunk_quiet)."""
        m, q = C.c_int(), C.c_int()
        self._check(self.lib.sparc_batch_tune(self.b, int(steps_per_trial),
                                              C.byref(m), C.byref(q)),
                    "sparc_batch_tune")
        return m.value, q.value

    def synchronize(self):
        self._check(self.lib.sparc_batch_synchronize(self.b),
                    "sparc_batch_synchronize")

    @property
    def stream(self):
        s = C.c_void_p()
        self._check(self.lib.sparc_batch_stream(self.b, C.byref(s)),
                    "sparc_batch_stream")
        return s.value

    @property
    def launch_count(self):
        n = C.c_int64()
        self._check(self.lib.sparc_batch_launch_count(self.b, C.byref(n)),
                    "sparc_batch_launch_count")
        return n.value
