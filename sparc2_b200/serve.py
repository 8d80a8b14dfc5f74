"""Python client of the serving loop (sparc_serve_* of include/sparc_gpu.h).

The server (C++, a worker thread over one batch) queues requests, admits
them by a device-memory budget and runs them as batch members.  This module
drives it the way a service front end would: requests arrive on a seeded
Poisson schedule and are submitted as they arrive; prefetch threads build
their host inputs (background arrays, source) in arrival order, a bounded
window ahead of admission; builder threads turn admitted requests into
SPARC_FP32 handles (the device set-up) while the batch keeps stepping; a
collector thread takes finished requests, reads their result and releases
their memory.  The reference has no counterpart.
"""
import ctypes as C
import threading
import time

import numpy as np

from . import abi
from .sim import Simulation


class Server:
    def __init__(self, capacity, budget_bytes, quantum=10, device=0):
        self.lib = abi.load()
        s = C.c_void_p()
        r = self.lib.sparc_server_create(int(device), int(capacity),
                                         int(budget_bytes), int(quantum),
                                         C.byref(s))
        if r != abi.SPARC_OK:
            raise abi.SparcError(r, "sparc_server_create", "")
        self.s = s
        self.device = device

    def _check(self, r, where):
        if r != abi.SPARC_OK:
            raise abi.SparcError(r, where,
                                 self.lib.sparc_server_last_error(self.s).decode())

    def close(self):
        if getattr(self, "s", None):
            self.lib.sparc_server_destroy(self.s)
            self.s = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, params, first, steps):
        t = C.c_int64()
        self._check(self.lib.sparc_serve_submit(self.s, C.byref(params),
                                                int(first), int(steps),
                                                C.byref(t)), "sparc_serve_submit")
        return t.value

    def next(self, state, timeout_s):
        """A not yet taken ticket in `state`, or None after timeout_s."""
        t = C.c_int64()
        r = self.lib.sparc_serve_next(self.s, int(state),
                                      int(timeout_s * 1000), C.byref(t))
        if r == abi.SPARC_ERR_TIMEOUT:
            return None
        self._check(r, "sparc_serve_next")
        return t.value

    def attach(self, ticket, sim):
        self._check(self.lib.sparc_serve_attach(self.s, int(ticket), sim.h),
                    "sparc_serve_attach")

    def result(self, ticket):
        """(state, times) of a DONE/FAILED ticket; times = submit, admit,
        start, done in seconds since the server started."""
        h = C.c_void_p()
        times = np.zeros(4)
        st = C.c_int()
        self._check(self.lib.sparc_serve_result(self.s, int(ticket),
                                                C.byref(h), abi.dptr(times),
                                                C.byref(st)),
                    "sparc_serve_result")
        return st.value, times

    def release(self, ticket):
        self._check(self.lib.sparc_serve_release(self.s, int(ticket)),
                    "sparc_serve_release")

    def stats(self):
        v = np.zeros(12)
        self._check(self.lib.sparc_serve_stats(self.s, abi.dptr(v)),
                    "sparc_serve_stats")
        keys = ["queued", "admitted", "running", "done", "budget_used",
                "max_concurrent", "batched_steps", "rounds", "point_updates",
                "worker_gpu_wait_s", "max_running", "joined_running"]
        return dict(zip(keys, v.tolist()))


def estimate_bytes(params):
    lib = abi.load()
    r, p = C.c_int64(), C.c_int64()
    lib.sparc_estimate_bytes(C.byref(params), C.byref(r), C.byref(p))
    return r.value, p.value


def drive(server, requests, build, on_result, builders=2, poll_s=0.05,
          horizon_s=None, deadline_s=None, prefetch=4, timings=None):
    """Runs a request stream through `server`.

    requests: list of (arrival_s, key, params, first, steps), sorted by
    arrival; build(key) -> (background, source) makes a request's host
    inputs; on_result(key, sim, state, times) sees each finished request
    before its handle is closed.  Requests arriving after horizon_s are not
    submitted.  prefetch: how many submitted requests may have their host
    inputs built ahead of admission (0: build after admission).  timings:
    an optional dict that receives, per key, the seconds spent building the
    host inputs and on the device set-up (sparc_create, background and
    source).  Raises TimeoutError if the stream has not drained deadline_s
    seconds after the start.  Returns the wall time from the start to the
    last result."""
    keys = {}
    lock = threading.Lock()
    done = threading.Event()
    submitted = [0]
    collected = [0]
    errors = []
    sims = {}
    # host inputs built ahead of admission: ticket -> [event, (bg, src)];
    # admission is first-in first-out, so building in submission order
    # always has the next admitted request's inputs first
    order = []
    inputs = {}
    window = threading.Semaphore(max(1, prefetch))
    cv = threading.Condition(lock)

    def host_inputs(tk, key):
        t = time.perf_counter()
        bg, src = build(key)
        if timings is not None:
            timings.setdefault(key, {})["host_build_s"] = time.perf_counter() - t
        return bg, src

    def prefetcher():
        while not done.is_set():
            with cv:
                while not order and not done.is_set():
                    cv.wait(poll_s)
                if done.is_set():
                    return
                tk = order.pop(0)
                key, _ = keys[tk]
            while not window.acquire(timeout=poll_s):
                if done.is_set():
                    return
            try:
                res = host_inputs(tk, key)
            except Exception as e:
                res = e
            with lock:
                inputs[tk][1] = res
            inputs[tk][0].set()

    def submitter():
        t0 = time.perf_counter()
        for arr, key, params, first, steps in requests:
            if horizon_s is not None and arr > horizon_s:
                break
            wait = arr - (time.perf_counter() - t0)
            if wait > 0 and done.wait(wait):
                return
            with lock:       # builders look the ticket up under this lock
                tk = server.submit(params, first, steps)
                keys[tk] = (key, params)
                submitted[0] += 1
                if prefetch > 0:
                    inputs[tk] = [threading.Event(), None]
                    order.append(tk)
                    cv.notify_all()
        with lock:
            submitted.append(True)    # marks the end of submissions

    def builder():
        while not done.is_set():
            tk = server.next(abi.SPARC_REQ_ADMITTED, poll_s)
            if tk is None:
                continue
            with lock:
                key, params = keys[tk]
            try:
                if prefetch > 0:
                    ev = inputs[tk][0]
                    while not ev.wait(poll_s):
                        if done.is_set():
                            return
                    with lock:
                        res = inputs.pop(tk)[1]
                    window.release()
                    if isinstance(res, Exception):
                        raise res
                    bg, src = res
                else:
                    bg, src = host_inputs(tk, key)
                t = time.perf_counter()
                sim = Simulation(params, bg, src, device=server.device)
                if timings is not None:
                    timings.setdefault(key, {})["device_setup_s"] = time.perf_counter() - t
                del bg
                with lock:
                    sims[tk] = sim
                server.attach(tk, sim)
            except Exception as e:           # give the budget back
                errors.append(e)
                server.release(tk)
                with lock:
                    collected[0] += 1

    def collector():
        while not done.is_set():
            tk = server.next(abi.SPARC_REQ_DONE, poll_s)
            if tk is not None:
                st, times = server.result(tk)
                with lock:
                    key, _ = keys[tk]
                    sim = sims.pop(tk)
                try:
                    on_result(key, sim, st, times)
                finally:
                    sim.close()
                    server.release(tk)
                    with lock:
                        collected[0] += 1
            with lock:
                finished = len(submitted) > 1 and collected[0] >= submitted[0]
            if finished:
                done.set()
                return

    t0 = time.perf_counter()
    threads = [threading.Thread(target=submitter, daemon=True)]
    threads += [threading.Thread(target=builder, daemon=True)
                for _ in range(builders)]
    if prefetch > 0:
        threads += [threading.Thread(target=prefetcher, daemon=True)
                    for _ in range(min(prefetch, 2))]
    threads.append(threading.Thread(target=collector, daemon=True))
    for t in threads:
        t.start()
    while not done.wait(0.1):
        if deadline_s is not None and time.perf_counter() - t0 > deadline_s:
            done.set()
            for t in threads:
                t.join(timeout=10 * poll_s + 1.0)
            raise TimeoutError("request stream did not drain in %g s: %s"
                               % (deadline_s, server.stats()))
    wall = time.perf_counter() - t0
    for t in threads:
        t.join(timeout=10 * poll_s + 1.0)
    if errors:
        raise errors[0]
    return wall
