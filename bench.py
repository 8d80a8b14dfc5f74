#!/usr/bin/env python
"""Benchmark of the SPARC linear wave time step on B200.

A step is one driver iteration (driver.f90:123-202): forcing, the five RK
stages, the diagnostics reduction and FILTER_VARS at its cadence.  The
workload is the plain MHD flux tube (256x256x300, FP64, 200 seeded PSR
pulses, dt = 0.5 s, CPML on six faces), the configuration the headline
grid-point-update rate is quoted on.  Prints one JSON line.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun (N > 1) every rank advances its own replica (the path does
not shard across GPUs here) and the time is the max over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from sparc2_b200 import abi, workloads as W  # noqa: E402

METRIC = "grid-pt updates/s"
UNIT = "grid-pt updates/s"
WORKLOAD = ("plain MHD flux tube 256x256x300 FP64 (100x100 Mm, z -25..+1 Mm, "
            "B0 3 kG, maxVA 40 km/s, CPML 10 pts on 6 faces, 200 seeded PSR "
            "pulses, dt 0.5 s, z filter every 10 / xy every 30 iterations)")
CPU_SAMPLE = (64, 64, 300)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=120)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="gpu", choices=["gpu", "reference"])
    ap.add_argument("--workload", default="cfg1",
                    choices=["cfg1", "cfg0", "ensemble", "serve"],
                    help="cfg1: MHD flux tube 256x256x300; cfg0: quiet-Sun "
                    "64x64x128; ensemble: 64 seeded FP32 members advanced by "
                    "the batched engine")
    ap.add_argument("--members", type=int, default=64,
                    help="ensemble size (ensemble workload)")
    ap.add_argument("--rate", type=float, default=5.0,
                    help="serve: Poisson arrival rate (requests/s)")
    ap.add_argument("--duration", type=float, default=60.0,
                    help="serve: seconds of arrivals")
    ap.add_argument("--steps-scale", type=float, default=0.05,
                    help="serve: request durations (500-4000 iterations) "
                    "scaled by this factor")
    ap.add_argument("--budget-gb", type=float, default=150.0,
                    help="serve: device-memory admission budget")
    ap.add_argument("--no-extras", action="store_true",
                    help="cfg1: skip the FP32 precision-form and batched-ensemble "
                    "lines that the default run adds beside the FP64 number")
    ap.add_argument("--no-fp64-compare", action="store_true",
                    help="ensemble: skip timing the FP64 plain cfg1 step")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"],
                    help="fp64: plain form; fp32: precision form (depth-scaled "
                    "FP32 state, compensated RK update)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serve", action="store_true",
                    help="cfg1: skip the bounded serving leg of the default run")
    ap.add_argument("--serve-rate", type=float, default=5.0,
                    help="cfg1 serving leg: arrivals per second")
    ap.add_argument("--serve-duration", type=float, default=30.0,
                    help="cfg1 serving leg: seconds of arrivals")
    ap.add_argument("--e2e-steps", type=int, default=60,
                    help="iterations between the state upload and read-back of "
                    "the end-to-end leg (the reference driver reads the state "
                    "back only at its output cadence, e.g. 1200 iterations)")
    ap.add_argument("--kernel-steps", type=int, default=10)
    ap.add_argument("--zchunk", type=int, default=0,
                    help="z extent of the stage work items (0: autotune)")
    ap.add_argument("--timed-only", action="store_true",
                    help="only the warm-up and the timed region (profiling)")
    ap.add_argument("--grid", type=int, nargs=3, default=None,
                    metavar=("NX", "NY", "NZ"),
                    help="same physics on a smaller grid (profiling only)")
    return ap.parse_args()


def algorithmic_bytes_per_point(p, with_filters=True):
    """Bytes per grid-point update of one RK step:
    w*[14V + 5C + 14*sum_faces(P*phi) + 2V/n_z + 2V/n_xy] (+2V words of
    the compensated-sum carry in the precision form); w word size,
    V state fields, C 3-D background inputs (quiet: 0, MHD: 6), P CPML
    fields per face, phi the fraction of points in that face's slab."""
    w = 8 if p.precision == abi.SPARC_FP64 else 4
    mhd = p.magnetic == 2
    V = 8 if mhd else 5
    C = 6 if mhd else (0 if p.magnetic == 0 and p.periodic else 5)
    P = 6 if mhd else 2
    phi = 0.0
    if p.use_pml or p.use_hpml:
        phi += (p.npml_zb + p.npml_zt) / p.nz
    if p.use_hpml:
        phi += (p.npml_xb + p.npml_xt) / p.nx + (p.npml_yb + p.npml_yt) / p.ny
    b = 14 * V + 5 * C + 14 * P * phi
    if w == 4:
        b += 2 * V  # compensated-sum carry, read and written by stage 5
    if with_filters:
        nz = int(np.floor(max(p.t_z, p.timestep) / p.timestep + 1e-5))
        nxy = int(np.floor(max(p.t_xy, p.timestep) / p.timestep + 1e-5))
        b += 2 * V / nz + 2 * V / nxy
    return w * b


def workload(name, precision=abi.SPARC_FP64, grid=None):
    fp = "FP64" if precision == abi.SPARC_FP64 else "FP32 precision form"
    if name == "cfg0":
        p, bg, src = W.cfg0(precision=precision)
        desc = ("plain quiet-Sun hydro 64x64x128 %s (50 Mm periodic, z -20..+1 "
                "Mm, z-CPML 10, v_z pulse 3 mHz, dt 1 s)" % fp)
        return p, bg, src, desc
    desc = WORKLOAD.replace("FP64", fp)
    if grid is None:
        p, bg, src = W.cfg1(precision=precision)
        return p, bg, src, desc
    nx, ny, nz = grid
    p, bg, src = W.cfg1(nx=nx, ny=ny, nz=nz, precision=precision,
                        length_mm=100.0 * nx / 256)
    return p, bg, src, desc


def p_V(p):
    return 8 if p.magnetic == 2 else 5


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", f"--id={index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        time.sleep(0.3)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except ValueError:
                continue
            for n, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus and args.impl == "gpu":
        print(f"warning: WORLD_SIZE={world} but --gpus {args.gpus}",
              file=sys.stderr)
    return world, rank, local


def cpu_baseline(steps=None, threads=None):
    """The oracle (C++/OpenMP FP64 restatement of the reference) on a
    64x64x300 sub-grid of the same physics, all host threads."""
    import oracle
    oracle.build()
    threads = threads or os.cpu_count()
    oracle.set_threads(threads)
    p, bg, src, _ = workload("cfg1", grid=CPU_SAMPLE)
    o = oracle.Oracle(p, bg, src)
    o.run(0, 1)                      # warm (first iteration doubles PSR)
    n = steps or 12
    t = time.perf_counter()
    o.run(1, n)
    dt = time.perf_counter() - t
    pts = p.nx * p.ny * p.nz
    return {"value": pts * n / dt, "unit": UNIT, "cores": threads,
            "kind": "port",
            "sample": (f"oracle (C++17/OpenMP FP64 restatement of the "
                       f"reference) on a {CPU_SAMPLE[0]}x{CPU_SAMPLE[1]}x"
                       f"{CPU_SAMPLE[2]} sub-grid of the same flux-tube "
                       f"physics, {n} driver iterations, {threads} threads")}


def run_reference(args, world, rank):
    """The reference arm: the oracle (the FP64 C++/OpenMP restatement of the
    reference; the Fortran/MPI reference cannot be built here) on the
    headline configuration itself, 256x256x300, with every host thread; one
    step is one driver iteration (about 6 s on 16 cores)."""
    if rank != 0:
        return
    import oracle
    oracle.build()
    threads = os.cpu_count()
    oracle.set_threads(threads)
    p, bg, src, desc = workload(args.workload if args.workload in ("cfg0", "cfg1")
                                else "cfg1", grid=args.grid)
    o = oracle.Oracle(p, bg, src)
    del bg
    # warm-up iterations; at least one, timed, to bound the run: the timed
    # iterations are capped so that they take about 150 s (a full-grid
    # iteration takes seconds), and the rate is per iteration run
    W = max(1, args.warmup)
    t = time.perf_counter()
    o.run(0, W)
    t_it = (time.perf_counter() - t) / W
    n = max(1, min(args.steps, int(150.0 / max(t_it, 1e-3))))
    t = time.perf_counter()
    o.run(W, n)
    dt = time.perf_counter() - t
    pts = p.nx * p.ny * p.nz
    v = pts * n / dt
    sample = (f"each step one driver iteration of the oracle (FP64 C++/OpenMP "
              f"restatement of the reference; the Fortran/MPI reference cannot "
              f"be built here) on the full {p.nx}x{p.ny}x{p.nz} grid of the "
              f"benchmark configuration, {threads} threads; {n} of the "
              f"{args.steps} steps timed (capped at about 150 s)")
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dt * 1e3 / n, "steps_timed": n, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded analytic background and pulse table)",
        "config": {"workload": desc, "grid": [p.nx, p.ny, p.nz],
                   "same_config": True},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads,
                         "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_gpu(args, world, rank, local):
    import torch
    from sparc2_b200 import Simulation
    from sparc2_b200.replicas import Replicas
    dev = local
    torch.cuda.set_device(dev)
    rep = Replicas("nccl")
    fp32 = args.precision == "fp32"
    prec = abi.SPARC_FP32 if fp32 else abi.SPARC_FP64
    wsize = 4 if fp32 else 8
    p, bg, src, desc = workload(args.workload, precision=prec, grid=args.grid)
    sim = Simulation(p, bg, src, device=dev)
    del bg
    pts = p.nx * p.ny * p.nz
    stream = torch.cuda.ExternalStream(sim.stream, device=dev)
    barrier = rep.barrier
    max_over_ranks = rep.max

    # the z extent of the stage work items is autotuned on real iterations
    # of the loop (untimed), then the warm-up iterations (graph capture
    # happens here) run
    W_ = args.warmup
    K = args.steps
    if args.zchunk > 0:
        sim.set_zchunk(args.zchunk)
        start, zchunk = 0, sim.zchunk
    else:
        start, zchunk = sim.tune(0, steps_per_trial=2)
    sim.run(start, W_)
    sim.synchronize()
    torch.cuda.synchronize(dev)
    clocks = Clocks(dev)
    n0 = sim.launch_count
    barrier()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.run(start + W_, K)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize(dev)
    barrier()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop() if clocks else None
    launches = sim.launch_count - n0
    d, status = sim.diagnostics()
    ms_max = max_over_ranks(ms)
    value = world * pts * K / (ms_max / 1e3)
    if args.timed_only:
        if rank == 0:
            print(json.dumps({"timed_only": True, "value": value,
                              "ms_per_step": ms_max / K}), flush=True)
        sim.close()
        rep.close()
        return

    # stage kernels alone (five fused RK-stage launches + the PSR forcing
    # of an iteration, no filter) for the roofline figure
    M = args.kernel_steps
    k0 = torch.cuda.Event(enable_timing=True)
    k1 = torch.cuda.Event(enable_timing=True)
    k0.record(stream)
    for nn in range(start + W_ + K, start + W_ + K + M):
        sim.step(nn)
    k1.record(stream)
    k1.synchronize()
    kms = k0.elapsed_time(k1) / M
    hbm, peak_kind = peaks()
    stage_bytes = algorithmic_bytes_per_point(p, with_filters=False) * pts
    achieved = stage_bytes / (kms / 1e3) / 1e9
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "stage_traffic.json")
    if os.path.exists(tfile):
        try:
            with open(tfile) as f:
                t = json.load(f)
            if t.get("workload") == args.workload + "_" + args.precision:
                traffic = t.get("bytes_per_step")
        except Exception:
            traffic = None

    # FILTER_VARS alone: an xy + z filter event (the fused y-then-x pass and
    # the z pass) on the current state, timed over a few events; algorithmic
    # bytes per event: a read and a write of the state per pass (2 passes),
    # plus the carry read of the first pass in the precision form
    F_EV = 5
    ev_xy = int(np.floor(max(p.t_xy, p.timestep) / p.timestep + 1e-5))
    ev_z = int(np.floor(max(p.t_z, p.timestep) / p.timestep + 1e-5))
    nn_f = ev_xy * ev_z  # an iteration on both cadences
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    sim.filter_vars(nn_f)
    f0.record(stream)
    for _ in range(F_EV):
        sim.filter_vars(nn_f)
    f1.record(stream)
    f1.synchronize()
    fms = f0.elapsed_time(f1) / F_EV
    fbytes = wsize * p_V(p) * pts * (4 + (1 if fp32 else 0))
    filt_roof = {"bound": "hbm", "achieved": fbytes / (fms / 1e3) / 1e9, "peak": hbm,
                 "unit": "GB/s", "frac": fbytes / (fms / 1e3) / 1e9 / hbm,
                 "peak_kind": peak_kind, "kernel": "one FILTER_VARS event (xy and z): "
                 "fused y-then-x pass + z pass", "algorithmic_bytes_per_launch": fbytes,
                 "ms_per_launch": fms}

    # end to end through the per-iteration C-ABI calls of the reference's
    # driver loop (STEP, norm readback, FILTER_VARS): state uploaded from
    # pinned host memory at the start, read back at the end, diagnostics
    # read back every iteration
    E = args.e2e_steps
    a_host, psi_host = sim.get_state()
    pin_a = torch.empty(a_host.size, dtype=torch.float64, pin_memory=True).numpy()
    pin_p = torch.empty(max(psi_host.size, 1), dtype=torch.float64,
                        pin_memory=True).numpy()
    pin_a[:] = a_host.ravel()
    pin_p[:psi_host.size] = psi_host
    first = start + W_ + K + M
    barrier()
    torch.cuda.synchronize(dev)
    x0 = torch.cuda.Event(enable_timing=True)
    x1 = torch.cuda.Event(enable_timing=True)
    x0.record(stream)
    sim.set_state(pin_a, pin_p[:psi_host.size] if psi_host.size else None)
    for nn in range(first, first + E):
        sim.step(nn)
        sim.diagnostics()
        sim.filter_vars(nn)
    sim.lib.sparc_get_state(sim.h, abi.dptr(pin_a), abi.dptr(pin_p))
    x1.record(stream)
    x1.synchronize()
    ems = max_over_ranks(x0.elapsed_time(x1))
    e2e = world * pts * E / (ems / 1e3)
    # bytes that cross PCIe: the device state is FP32 in the precision form
    # (its compensated-sum carry is read back with it)
    h2d = (wsize * (a_host.size + psi_host.size) + 8 * E) / E
    d2h = (wsize * (a_host.size * (2 if fp32 else 1) + psi_host.size)
           + 40 * E) / E

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline()

    # the precision comparison: the FP32 precision form and the FP32
    # batched ensemble on the same GPU, beside this FP64 plain number
    extras = {}
    if (world == 1 and not args.no_extras and args.workload == "cfg1"
            and not fp32 and args.grid is None):
        sim.close()
        sim = None
        extras["fp32_precision_form"] = measure_fp32_cfg2(dev)
        extras["fp32_precision_form"]["ratio_vs_fp64_plain"] = \
            extras["fp32_precision_form"]["value"] / value
        extras["fp32_precision_form"]["error_vs_oracle"] = fp32_errors(dev)
        extras["fp32_batched"] = measure_ensemble(dev, members=args.members)
        extras["fp32_batched"]["ratio_vs_fp64_plain"] = \
            extras["fp32_batched"]["value"] / value
        extras["fp32_batched"]["error_vs_oracle"] = fp32_errors(dev, batched=True)
        if not args.no_serve:
            sv, _, rec, _, _ = measure_serve(dev, args.serve_rate, args.serve_duration,
                                             args.steps_scale, args.budget_gb)
            rec["ratio_vs_fp64_plain"] = sv / value
            extras["fp32_served"] = rec

    if rank != 0:
        if sim is not None:
            sim.close()
        rep.close()
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": K, "warmup": W_, "ms_per_step": ms_max / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if fp32 else "f64",
        "data": "synthetic (seeded analytic background and "
        "pulse table; no public dataset)",
        "config": {"workload": desc, "grid": [p.nx, p.ny, p.nz],
                   "precision": "fp32 precision form" if fp32 else "fp64 plain",
                   "zchunk": zchunk,
                   "zchunk_note": ("z extent of the stage work items, autotuned on "
                                   "%d untimed iterations before the warm-up" % start)
                   if args.zchunk <= 0 else "z extent of the stage work items, set",
                   "parallelism": "replicas" if world > 1 else "single GPU",
                   "l2": "working set %.1f GB > 126 MB L2 (no flush needed)"
                   % (3 * p_V(p) * wsize * pts / 1e9)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm,
                     "unit": "GB/s", "frac": achieved / hbm,
                     "peak_kind": peak_kind, "traffic": traffic,
                     "kernel": "5 fused RK-stage launches + PSR forcing of "
                     "one iteration",
                     "algorithmic_bytes_per_launch": stage_bytes,
                     "ms_per_launch": kms},
        "filter_roofline": filt_roof,
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "steps": E,
                "pattern": "state uploaded from pinned host memory, then per "
                "iteration sparc_step, sparc_diagnostics read back (the "
                "reference's per-iteration norm) and sparc_filter_vars; state "
                "and CPML fields read back after the %d iterations" % E},
        "gpu_launches": launches,
        "diag": {"ke_norm": d.ke_norm, "iteration": d.iteration,
                 "status": int(status)},
    }
    if clk:
        line["clocks"] = clk
    if cpu:
        line["cpu_baseline"] = cpu
    line.update(extras)
    print(json.dumps(line), flush=True)
    if sim is not None:
        sim.close()
    rep.close()


def fp64_plain_rate(dev, steps=20, warmup=3):
    """The FP64 plain form on the flux-tube configuration (256x256x300),
    timed with CUDA events on its stream: the comparison point of the
    batched precision form on the same GPU."""
    import torch
    from sparc2_b200 import Simulation
    p, bg, src, _ = workload("cfg1")
    sim = Simulation(p, bg, src, device=dev)
    del bg
    stream = torch.cuda.ExternalStream(sim.stream, device=dev)
    start, _ = sim.tune(0, steps_per_trial=2)
    sim.run(start, warmup)
    sim.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.run(start + warmup, steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    sim.close()
    return p.nx * p.ny * p.nz / (ms / 1e3), ms


def fp32_errors(dev, batched=False):
    """Errors of the precision form against the FP64 oracle: the flux-tube
    physics on 96x96x300 columns (the committed oracle fixture
    tests/golden/fluxtube_96x96x300.npz, 1000 iterations from rest), run
    alone or as a member of the batched engine.  Per field, the relative L2
    and the max-norm error (relative to max |oracle|) over the fixture's
    strided sample of the state at iterations 100, 500 and 1000."""
    from sparc2_b200 import Simulation
    from sparc2_b200.batch import Batch
    from tests.golden import make_fluxtube_1000 as F
    path = os.path.join(ROOT, "tests", "golden", F.NAME + ".npz")
    if not os.path.exists(path):
        return None
    ref = np.load(path)
    p, bg, src = F.config()
    p.precision = abi.SPARC_FP32
    sim = Simulation(p, bg, src, device=dev)
    del bg
    out = {}
    done = 0
    batch = Batch(1, device=dev) if batched else None
    for it in F.CHECKPOINTS:
        if batched:
            q = batch.add(sim, done, it - done)
            batch.run(it - done)
            batch.synchronize()
            batch.remove(q)
        else:
            sim.run(done, it - done)
        done = it
        a, psi = sim.get_state()
        samp = F.sample(a, psi)["samp"]
        rl2, mx = [], []
        for l in range(samp.shape[0]):
            o = ref[f"it{it}_samp"][l]
            g = samp[l]
            den = np.sqrt(np.sum(o * o))
            rl2.append(float(np.sqrt(np.sum((g - o) ** 2)) / den) if den > 0 else 0.0)
            m = np.max(np.abs(o))
            mx.append(float(np.max(np.abs(g - o)) / m) if m > 0 else 0.0)
        out[str(it)] = {"rel_l2": rl2, "max_norm": mx,
                        "max_rel_l2": max(rl2), "max_max_norm": max(mx)}
    if batch is not None:
        batch.close()
    sim.close()
    return {"against": "FP64 oracle fixture, flux tube 96x96x300 (37.5 Mm, "
            "CPML 10 on 6 faces, 200 seeded PSR pulses), 1000 iterations from "
            "rest%s" % (", run as a batch member" if batched else ""),
            "fields": ["rho", "vx", "vy", "vz", "p", "bx", "by", "bz"],
            "sample": "every %dth value of each field" % F.STRIDE,
            "iterations": out}


def measure_fp32_cfg2(dev, steps=40, warmup=3):
    """The precision form on the flux-tube configuration (cfg2), timed like
    the headline: graph-launched iterations, CUDA events on its stream."""
    import torch
    from sparc2_b200 import Simulation
    p, bg, src, desc = workload("cfg1", precision=abi.SPARC_FP32)
    sim = Simulation(p, bg, src, device=dev)
    del bg
    stream = torch.cuda.ExternalStream(sim.stream, device=dev)
    start, zchunk = sim.tune(0, steps_per_trial=2)
    sim.run(start, warmup)
    sim.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.run(start + warmup, steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    sim.close()
    pts = p.nx * p.ny * p.nz
    return {"value": pts / (ms / 1e3), "unit": UNIT, "ms_per_step": ms, "steps": steps,
            "dtype": "f32", "zchunk": zchunk, "workload": desc}


def measure_ensemble(dev, members=64, steps=100, warmup=2):
    """The batched precision form: `members` seeded FP32 simulations through
    the batched engine (autotuned z extents), one graph launch per step."""
    import torch
    from sparc2_b200 import Simulation
    from sparc2_b200.batch import Batch
    draws = W.ensemble_draws(members)
    sims, pts = [], 0
    t0 = time.perf_counter()
    for nx, nz, b0, depth in draws:
        p, bg, src = W.member(nx, nz, b0, depth)
        sims.append(Simulation(p, bg, src, device=dev))
        pts += p.nx * p.ny * p.nz
        del bg
    setup = time.perf_counter() - t0
    batch = Batch(len(sims), device=dev)
    for sm in sims:
        batch.add(sm, 0, 1000)
    stream = torch.cuda.ExternalStream(batch.stream, device=dev)
    tiles = batch.tune(steps_per_trial=1)
    batch.run(warmup)
    batch.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    batch.run(steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    batch.close()
    for sm in sims:
        sm.close()
    nq = sum(1 for d in draws if d[2] <= 0)
    return {"value": pts / (ms / 1e3), "unit": UNIT, "ms_per_step": ms, "steps": steps,
            "dtype": "f32", "members": len(draws), "quiet_members": nq,
            "grid_points": pts, "tiles": {"zchunk_mhd": tiles[0], "zchunk_quiet": tiles[1],
                      "mhd_tile": [32, 8]},
            "setup_s": setup,
            "workload": "batched ensemble: %d seeded members (nx=ny in {96..256}, nz in "
                        "[150, 300], quiet or flux tube, one pulse each), a step advances "
                        "every member one driver iteration" % len(draws)}


def run_ensemble(args, world, rank, local):
    """Batched precision form: `members` seeded FP32 simulations of uneven
    grids (quiet and flux-tube) advanced together by the batched engine,
    one CUDA-graph launch per step; a step advances every member by one
    driver iteration."""
    import torch
    from sparc2_b200 import Simulation
    from sparc2_b200.batch import Batch
    from sparc2_b200.replicas import Replicas
    dev = local
    torch.cuda.set_device(dev)
    rep = Replicas("nccl")
    draws = W.ensemble_draws(args.members)
    W_, K, E = args.warmup, args.steps, args.e2e_steps
    total_steps = 1000
    sims, params = [], []
    t_setup = time.perf_counter()
    for nx, nz, b0, depth in draws:
        p, bg, src = W.member(nx, nz, b0, depth)
        sims.append(Simulation(p, bg, src, device=dev))
        params.append(p)
        del bg
    t_setup = time.perf_counter() - t_setup
    pts = sum(p.nx * p.ny * p.nz for p in params)
    batch = Batch(len(sims), device=dev)
    for s in sims:
        batch.add(s, 0, total_steps)
    stream = torch.cuda.ExternalStream(batch.stream, device=dev)
    tiles = batch.tune(steps_per_trial=2)
    tuned_steps = 1000 - int(batch.remaining()[0])
    batch.run(W_)
    batch.synchronize()
    clocks = Clocks(dev)
    n0 = batch.launch_count
    rep.barrier()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    batch.run(K)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize(dev)
    rep.barrier()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop() if clocks else None
    launches = batch.launch_count - n0
    ms_max = rep.max(ms)
    value = world * pts * K / (ms_max / 1e3)
    hbm, peak_kind = peaks()
    step_bytes = sum(algorithmic_bytes_per_point(p) * p.nx * p.ny * p.nz
                     for p in params)
    achieved = step_bytes / (ms_max / K / 1e3) / 1e9
    diags = [s.diagnostics() for s in sims]
    unstable = sum(1 for _, r in diags if r != abi.SPARC_OK)

    # end to end through the public API: every member restarts from a state
    # uploaded from pinned host memory (set_state, outside the batch), E
    # batched steps with every member's diagnostics read back each step,
    # every member's state read back into pinned host memory at the end
    for q in list(batch.members):
        batch.remove(q)
    sizes = [(s.n_state, s.n_psi) for s in sims]
    big = max(n + m for n, m in sizes)
    pin = torch.zeros(big, dtype=torch.float64, pin_memory=True).numpy()
    first = int(diags[0][0].iteration) + 1
    rep.barrier()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for s, (n, m) in zip(sims, sizes):
        pin[:n + m] = 0.0
        s.set_state(pin[:n], pin[n:n + m] if m else None)
        batch.add(s, first, E)
    for _ in range(E):
        batch.run(1)
        for s in sims:
            s.diagnostics()
    for q in list(batch.members):
        batch.remove(q)
    for s, (n, m) in zip(sims, sizes):
        s.lib.sparc_get_state(s.h, abi.dptr(pin[:n]), abi.dptr(pin[n:n + m]))
    torch.cuda.synchronize(dev)
    et = rep.max(time.perf_counter() - t0)
    e2e = world * pts * E / et
    n_state = sum(n for n, _ in sizes)
    n_psi = sum(m for _, m in sizes)
    # the device state is FP32: 4 bytes per value up, state + carry down
    h2d = 4 * (n_state + n_psi) / E
    d2h = (4 * (2 * n_state + n_psi) + 40 * len(sims) * E) / E
    batch.close()
    for s in sims:
        s.close()
    sims = None
    fp64 = None
    if rank == 0 and not args.no_fp64_compare:
        v64, ms64 = fp64_plain_rate(dev)
        fp64 = {"value": v64, "unit": UNIT, "ms_per_step": ms64,
                "workload": "plain MHD flux tube 256x256x300 FP64, one "
                "simulation (sparc_run, CUDA graphs), same GPU"}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline()
    if rank != 0:
        rep.close()
        return
    nq = sum(1 for d in draws if d[2] <= 0)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": K, "warmup": W_, "ms_per_step": ms_max / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded analytic backgrounds and "
        "sources; no public dataset)",
        "config": {"workload": "batched ensemble, FP32 precision form: %d "
                   "members (%d quiet, %d flux tube), nx=ny in {96..256}, nz "
                   "in [150, 300], one Gaussian source each, dt 0.5 s; a step "
                   "advances every member one driver iteration"
                   % (len(draws), nq, len(draws) - nq),
                   "members": len(draws), "grid_points": pts,
                   "tiles": {"zchunk_mhd": tiles[0], "zchunk_quiet": tiles[1],
                             "mhd_tile": [32, 8],
                             "autotuner_steps": tuned_steps},
                   "setup_s": t_setup,
                   "parallelism": "replicas" if world > 1 else "single GPU",
                   "l2": "working set %.0f GB > 126 MB L2 (no flush needed)"
                   % (step_bytes / 1e9)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm,
                     "unit": "GB/s", "frac": achieved / hbm,
                     "peak_kind": peak_kind, "traffic": None,
                     "kernel": "one batched step (forcing, 5 persistent RK "
                     "stage launches, filter passes at cadence)",
                     "algorithmic_bytes_per_launch": step_bytes,
                     "ms_per_launch": ms_max / K},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "steps": E},
        "gpu_launches": launches,
        "diag": {"unstable_members": unstable},
    }
    if fp64:
        line["fp64_plain"] = fp64
        line["speedup_vs_fp64_plain"] = value / fp64["value"]
    if clk:
        line["clocks"] = clk
    if cpu:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)
    rep.close()


def measure_serve(dev, rate, duration, steps_scale, budget_gb=150.0):
    """Served solves, FP32: seeded Poisson arrivals at `rate` per second for
    `duration` seconds, request durations scaled by steps_scale, through
    the serving loop (budget admission into the running batch).  Returns
    (served rate, stats, the serve record)."""
    from sparc2_b200.serve import Server, drive
    draws = W.serve_draws(rate, duration, steps_scale=steps_scale)
    reqs = []
    for d in draws:
        p = W.member_params(d["nx"], d["nz"], d["B0"])
        reqs.append((d["arrival"], d["key"], p, 0, d["steps"]))
    res = {}
    timings = {}

    def build(key):
        _, bg, src = W.serve_request(draws[key])
        return bg, src

    def on_result(key, sim, state, times):
        d, _ = sim.diagnostics()
        res[key] = (state, times.copy(), d.ke_norm)

    srv = Server(capacity=64, budget_bytes=int(budget_gb * 1e9), quantum=10, device=dev)
    # a build (sparc_create, background and source set-up beside the running
    # batch) mostly waits on synchronisations: twelve builders overlap them
    wall = drive(srv, reqs, build, on_result, builders=12, prefetch=8, timings=timings,
                 deadline_s=20 * duration + 600)
    st = srv.stats()
    srv.close()
    lat = np.array([t[3] - t[0] for _, t, _ in res.values()])
    wait = np.array([t[1] - t[0] for _, t, _ in res.values()])
    setup = np.array([t[2] - t[1] for _, t, _ in res.values()])
    serv = np.array([t[3] - t[2] for _, t, _ in res.values()])
    hb = np.array([v["host_build_s"] for v in timings.values() if "host_build_s" in v])
    ds = np.array([v["device_setup_s"] for v in timings.values() if "device_setup_s" in v])
    pu = st["point_updates"]
    offered = sum(d["nx"] * d["nx"] * d["nz"] * d["steps"] for d in draws)
    pct = lambda a, q: float(np.percentile(a, q)) if a.size else None
    rec = {"p50_latency_s": pct(lat, 50), "p99_latency_s": pct(lat, 99),
           "p50_queue_wait_s": pct(wait, 50), "p99_queue_wait_s": pct(wait, 99),
           "p50_setup_s": pct(setup, 50), "p99_setup_s": pct(setup, 99),
           "p50_host_input_build_s": pct(hb, 50),
           "p50_device_setup_s": pct(ds, 50),
           "p50_service_s": pct(serv, 50), "p99_service_s": pct(serv, 99),
           "offered_point_updates_per_s": offered / duration,
           "served_point_updates": pu, "served_rate": pu / wall, "wall_s": wall,
           "requests": len(draws), "completed": len(res),
           "max_concurrent": st["max_concurrent"],
           "max_running_together": st["max_running"],
           "joined_running_batch": st["joined_running"],
           "worker_gpu_wait_s": st["worker_gpu_wait_s"],
           "workload": "served solves, FP32: Poisson arrivals at %g/s for %g s, "
           "nx=ny in [64,256], nz in [128,300], quiet or flux tube (B0 0.5-3 kG), "
           "one pulse or 50-500 PSR pulses, 500-4000 iterations x %g"
           % (rate, duration, steps_scale),
           "note": "latency = done - submit; set-up = start - admit (the admitted "
           "request's device set-up and attach; host inputs are built ahead of "
           "admission); the offered load is several times what one B200 serves"}
    return pu / wall, st, rec, len(draws), len(res)


def run_serve(args, world, rank, local):
    """Served solves, FP32: Poisson arrivals (seeded) of requests with
    random grid, background, source and duration, admitted by a device
    memory budget into the running batch; latency percentiles beside the
    served grid-point update rate."""
    import torch
    from sparc2_b200.replicas import Replicas
    dev = local
    torch.cuda.set_device(dev)
    rep = Replicas("nccl")
    clocks = Clocks(dev)
    value, st, rec, nreq, ndone = measure_serve(dev, args.rate, args.duration,
                                                args.steps_scale, args.budget_gb)
    clk = clocks.stop() if clocks else None
    if rank != 0:
        rep.close()
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": int(st["batched_steps"]), "warmup": 0,
        "ms_per_step": 1e3 * st["worker_gpu_wait_s"] / max(1, st["batched_steps"]),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded request stream)",
        "config": {"workload": "served solves, FP32: Poisson arrivals at %g/s "
                   "for %g s, nx=ny in [64,256], nz in [128,300], quiet or "
                   "flux tube (B0 0.5-3 kG), one pulse or 50-500 PSR pulses, "
                   "500-4000 iterations x %g" % (args.rate, args.duration,
                                                  args.steps_scale),
                   "requests": nreq, "completed": ndone,
                   "budget_gb": args.budget_gb, "slots": 64, "quantum": 10},
        "serve": rec,
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": None,
                "d2h_bytes_per_step": None,
                "note": "the served rate is end to end: host background "
                "generation, set-up, admission and result read-back inside"},
        "gpu_launches": None,
    }
    if clk:
        line["clocks"] = clk
    print(json.dumps(line), flush=True)
    rep.close()


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    if args.workload == "ensemble":
        run_ensemble(args, world, rank, local)
        return
    if args.workload == "serve":
        run_serve(args, world, rank, local)
        return
    run_gpu(args, world, rank, local)


if __name__ == "__main__":
    main()
