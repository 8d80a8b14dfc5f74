"""Seeded synthetic workloads: run parameters, backgrounds and sources.

No public dataset is involved.  The backgrounds are analytic (a polytrope
with an isothermal atmosphere, optionally threaded by a self-similar flux
tube) and every random draw comes from numpy's counter-based Philox
generator keyed by one documented 64-bit seed, so the oracle and the device
see identical inputs.

Array convention: numpy C-order shape (nz, ny, nx), which is the Fortran
(nx, ny, nz) layout of the reference (x fastest).
"""
import ctypes as C

import numpy as np

from . import abi

RSUN = 69598946770.0          # all_modules.f90:56
PI_REF = 3.14159265358979     # all_modules.f90:56
MM = 1.0e8                    # cm per Mm

SEED_CFG0 = 0x5A5C0000
SEED_CFG1 = 0x5A5C0001
SEED_CFG3 = 0x5A5C0003
SEED_CFG4 = 0x5A5C0004


def base_params(nx, ny, nz, *, magnetic=0, periodic=True, hpml=False,
                xlength=50.0 * MM, ylength=50.0 * MM, timestep=1.0,
                t_z=10.0, t_xy=30.0, npml=10, blocks=(2, 2, 4),
                maxva=4.0e6, precision=abi.SPARC_FP64):
    """sparc_params with the reference's sample .trol values
    (sparc_parameters:99-174) unless overridden."""
    p = abi.SparcParams()
    p.nx, p.ny, p.nz = nx, ny, nz
    p.magnetic = magnetic
    p.periodic = 1 if periodic else 0
    p.use_pml = 1
    p.use_hpml = 1 if hpml else 0
    p.stabilise = 1
    p.filter_mode_xy = 1
    p.filter_mode_z = 1
    p.block_x, p.block_y, p.block_z = blocks
    nh = npml if hpml else 0
    p.npml_xb = p.npml_xt = p.npml_yb = p.npml_yt = nh
    p.npml_zb = p.npml_zt = npml
    for f in ("pml_xb", "pml_xt", "pml_yb", "pml_yt"):
        getattr(p, f)[:] = (15.0, 3.0, 8.0, 0.1)
    for f in ("pml_zb", "pml_zt"):
        getattr(p, f)[:] = (5.0, 2.0, 8.0, 0.1)
    p.xlength, p.ylength = xlength, ylength
    p.timestep = timestep
    p.s_xy = p.s_z = 1.0
    p.t_xy, p.t_z = t_xy, t_z
    p.maxva = maxva
    p.sp_str, p.sp_length, p.sp_decay = 0.0, 10.0 * MM, 0.008
    p.precision = precision
    return p


def polytrope_1d(zaxis_mm, m=1.5, g=2.74e4, rho_s=2.0e-7, p_s=1.2e5,
                 gamma=5.0 / 3.0):
    """Adiabatic polytrope of index m below z = 0 with an isothermal layer
    above, in hydrostatic balance under constant gravity g (cgs)."""
    z = np.asarray(zaxis_mm, dtype=np.float64) * MM
    za = (m + 1.0) * p_s / (rho_s * g)      # polytropic length scale
    H = p_s / (rho_s * g)                   # isothermal scale height
    d = np.maximum(-z, 0.0)
    rho = np.where(z <= 0.0, rho_s * (1.0 + d / za) ** m,
                   rho_s * np.exp(-np.maximum(z, 0.0) / H))
    pre = np.where(z <= 0.0, p_s * (1.0 + d / za) ** (m + 1.0),
                   p_s * np.exp(-np.maximum(z, 0.0) / H))
    dlnrho = np.where(z <= 0.0, -m / (za + d), -1.0 / H)
    cs = np.sqrt(gamma * pre / rho)
    grav = np.full_like(z, g)
    return rho, pre, cs, grav, dlnrho


def quiet_background(nx, ny, nz, z_bot=-20.0, z_top=1.0, **kw):
    """Horizontally uniform polytrope background (3-D replicated arrays)."""
    zaxis = np.linspace(z_bot, z_top, nz)
    rho, pre, cs, grav, _ = polytrope_1d(zaxis, **kw)
    shape = (nz, ny, nx)
    bg = dict(
        rho0=np.ascontiguousarray(np.broadcast_to(rho[:, None, None], shape)),
        pre0=np.ascontiguousarray(np.broadcast_to(pre[:, None, None], shape)),
        cs0=np.ascontiguousarray(np.broadcast_to(cs[:, None, None], shape)),
        bx0=None, by0=None, bz0=None,
        zaxis=zaxis, grav=grav)
    return bg


def fluxtube_background(nx, ny, nz, xlength, ylength, z_bot=-25.0,
                        z_top=1.0, B0=3000.0, R0_mm=3.0, gamma=5.0 / 3.0,
                        periodic=False, p_floor=0.1):
    """Self-similar axisymmetric flux tube in the polytrope.

    B_z = Ba(z) exp(-r^2/R^2), R(z) = R0 (rho(z)/rho(0))^(-1/4), with the
    axis field Ba = B0 (R0/R)^2 so the tube flux is conserved; div B = 0
    then gives B_r = Ba (R'/R) r exp(-r^2/R^2).  The gas pressure is lowered
    by |B|^2/8pi for lateral balance, smoothly floored at p_floor*p (the
    3 kG surface field exceeds the photospheric gas pressure), and the
    density is lowered in proportion so the sound speed keeps its
    background value."""
    zaxis = np.linspace(z_bot, z_top, nz)
    rho, pre, cs, grav, dlnrho = polytrope_1d(zaxis, gamma=gamma)
    rho_s = np.interp(0.0, zaxis, rho)
    R = R0_mm * MM * (rho / rho_s) ** (-0.25)
    Rp_over_R = -0.25 * dlnrho
    Ba = B0 * (R0_mm * MM / R) ** 2
    if periodic:
        xs = np.arange(nx) / nx * xlength
        ys = np.arange(ny) / ny * ylength
    else:
        xs = np.arange(nx) / (nx - 1) * xlength
        ys = np.arange(ny) / (ny - 1) * ylength
    x = xs - 0.5 * xlength
    y = ys - 0.5 * ylength
    # exp(-r^2/R^2) = exp(-x^2/R^2) exp(-y^2/R^2): nz*(nx + ny) exponentials
    # instead of one per point; the cube is built by products, in place
    iR2 = 1.0 / (R * R)
    ex = np.exp(-(x * x)[None, :] * iR2[:, None])          # (nz, nx)
    ey = np.exp(-(y * y)[None, :] * iR2[:, None])          # (nz, ny)
    bz = (Ba[:, None] * ey)[:, :, None] * ex[:, None, :]
    bx = bz * (Rp_over_R[:, None, None] * x[None, None, :])
    by = bz * (Rp_over_R[:, None, None] * y[None, :, None])
    pm = bx * bx
    pm += by * by
    pm += bz * bz
    pm /= 8.0 * np.pi
    fac = pm                                      # q = 1 - pm/p, in place
    fac /= -pre[:, None, None]
    fac += 1.0
    lo = 2.0 * p_floor
    low = fac < lo                                # the floor only where it applies
    fac[low] = p_floor + p_floor * np.exp((fac[low] - lo) / p_floor)
    pre3 = fac * pre[:, None, None]
    rho3 = fac
    rho3 *= rho[:, None, None]
    cs3 = np.sqrt(gamma * pre3 / rho3)
    c = np.ascontiguousarray
    return dict(rho0=c(rho3), pre0=c(pre3), cs0=c(cs3), bx0=c(bx),
                by0=c(by), bz0=c(bz), zaxis=zaxis, grav=grav)


def pulse_source(*, amp=1.0e4, freq=3.0e-3, t1=300.0, st=75.0, px=25.0 * MM,
                 py=25.0 * MM, pz=-0.5 * MM, sr=0.5 * MM, sz=0.5 * MM,
                 direction=3, init=0):
    """A PULSE = 1 source (driver.f90:140-145), .trol units."""
    s = abi.SparcSource()
    s.kind = abi.SPARC_SRC_PULSE
    s.dir = direction
    s.init = init
    s.amp, s.t0, s.t1, s.st = amp, 1.0 / freq, t1, st
    s.px, s.py, s.pz, s.sr, s.sz = px, py, pz, sr, sz
    return s


def psr_table(params, npulses, seed, init=0):
    """Pulse table of PULSE = 2 drawn as RUN_PSR_PULSE does at its first call
    (all_modules.f90:539-588), from Philox uniforms instead of the
    system-clock-seeded RANDOM_NUMBER.  Returns a (npulses,) structured
    float64 array with the sparc_pulse fields."""
    nx, ny = params.nx, params.ny
    periodic = bool(params.periodic)
    rng = np.random.Generator(np.random.Philox(key=seed))
    T1 = 1.0 - rng.random((9, npulses))   # in (0, 1]: LOG() stays finite
    dx = 1.0 / nx if periodic else 1.0 / (nx - 1)
    dy = 1.0 / ny if periodic else 1.0 / (ny - 1)
    diml = RSUN
    mu_sr = 1.5 * max(dx, dy)
    sigma_sr = 0.2 * mu_sr
    mu_freq, sigma_freq = 3.3e-3, 0.5e-3
    nxb, nxt = (params.npml_xb, params.npml_xt) if params.use_hpml else (0, 0)
    nyb, nyt = (params.npml_yb, params.npml_yt) if params.use_hpml else (0, 0)
    px = nxb * 1.0 / nx + T1[0] * (nx - nxt - nxb) * 1.0 / nx
    py = nyb * 1.0 / ny + T1[1] * (ny - nyt - nyb) * 1.0 / ny
    pz = 1.0 - 0.1e8 / diml - T1[2] * (1.9e8 / diml)
    mu_sz = 0.05e8 / diml + 0.05e8 / diml / 2.0e8 * (1.0 - pz)
    sigma_sz = 0.2 * mu_sz
    r = np.sqrt(-2.0 * np.log(T1[3]))
    sr = mu_sr + sigma_sr * r * np.cos(2.0 * PI_REF * T1[4])
    sz = mu_sz + sigma_sz * r * np.sin(2.0 * PI_REF * T1[4])
    amp = 1.0e-1 + 0.2 * 1.0e-1 * np.sqrt(-2.0 * np.log(T1[5])) * \
        np.cos(2.0 * PI_REF * T1[6])
    t0 = 1.0 / (mu_freq + sigma_freq * np.sqrt(-2.0 * np.log(T1[7])) *
                np.cos(2.0 * PI_REF * T1[8]))
    psr_st = 120.0
    t1 = init * params.timestep + (3.0 + 1.0 * T1[6]) * psr_st
    tab = np.zeros(npulses, dtype=[(f, "f8") for f in
                                   ("px", "py", "pz", "sr", "sz", "amp",
                                    "t0", "t1")])
    tab["px"], tab["py"], tab["pz"] = px, py, pz
    tab["sr"], tab["sz"], tab["amp"] = sr, sz, amp
    tab["t0"], tab["t1"] = t0, t1
    return tab


def random_series(params, maxtime, cadforcing, seed):
    """A seeded stand-in for the forcingfunc cube of PULSE = 0 (the
    reference reads it from a FITS file): nx*ny*num_steps unit-variance
    samples, x fastest, with num_steps as driver.f90:38-39 sizes it for a
    run of `maxtime` iterations."""
    ns = int(np.floor(maxtime * params.timestep / cadforcing)) + 2
    ns = 2 * (ns // 2) + 2
    rng = np.random.Generator(np.random.Philox(key=seed))
    return np.ascontiguousarray(rng.standard_normal((ns, params.ny, params.nx)))


def random_source(series, *, cadforcing=30.0, ampl=1.0e3, depth=-0.15 * MM,
                  sigma=0.1 * MM, init=0):
    """A PULSE = 0 source (driver.f90:73-81, 130-132) over a forcing series of
    shape (num_steps, ny, nx); keeps the series alive on the returned object
    (attribute _keep).  ampl, depth, sigma: randomexciteampl (cm/s),
    randomexcitedepth and randomexcitesigma (cm)."""
    arr = np.ascontiguousarray(series, dtype=np.float64)
    s = abi.SparcSource()
    s.kind = abi.SPARC_SRC_RANDOM
    s.dir = 3
    s.init = init
    s.cadforcing, s.rnd_ampl = cadforcing, ampl
    s.rnd_depth, s.rnd_sigma = depth, sigma
    s.nseries = arr.shape[0]
    s.series = arr.ctypes.data_as(C.POINTER(C.c_double))
    s._keep = arr
    return s


def psr_source(table, direction=3, init=0, psr_st=120.0):
    """A PULSE = 2 source over a pulse table; keeps the table alive on the
    returned object (attribute _keep)."""
    s = abi.SparcSource()
    s.kind = abi.SPARC_SRC_PSR
    s.dir = direction
    s.init = init
    s.psr_st = psr_st
    arr = (abi.SparcPulse * len(table))()
    for n, row in enumerate(table):
        for f in ("px", "py", "pz", "sr", "sz", "amp", "t0", "t1"):
            setattr(arr[n], f, float(row[f]))
    s.npulses = len(table)
    s.pulses = arr
    s._keep = arr
    return s


# ------------------------------------------------------------- presets

def cfg0(nx=64, ny=64, nz=128, precision=abi.SPARC_FP64, blocks=(2, 2, 4)):
    """Plain quiet-Sun hydro: 64x64x128, 50 Mm periodic, z -20..+1 Mm,
    z-filter every 10 steps, xy-filter every 30, 10-point CPML top and
    bottom, dt = 1 s; the reference's v_z pulse at 3 mHz."""
    p = base_params(nx, ny, nz, magnetic=0, periodic=True, hpml=False,
                    xlength=50.0 * MM, ylength=50.0 * MM, timestep=1.0,
                    t_z=10.0, t_xy=30.0, blocks=blocks, precision=precision)
    bg = quiet_background(nx, ny, nz, -20.0, 1.0)
    src = pulse_source(px=0.5 * p.xlength, py=0.5 * p.ylength)
    return p, bg, src


def cfg1(nx=256, ny=256, nz=300, npulses=200, seed=SEED_CFG1,
         precision=abi.SPARC_FP64, blocks=(2, 2, 4), length_mm=100.0):
    """Plain MHD flux tube: 256x256x300 over 100x100 Mm, z -25..+1 Mm, CPML
    on all six faces, Alfven speed capped at 40 km/s, 200 seeded PSR
    pulses, dt = 0.5 s, z-filter every 10 steps and xy-filter every 30."""
    L = length_mm * MM
    p = base_params(nx, ny, nz, magnetic=2, periodic=False, hpml=True,
                    xlength=L, ylength=L, timestep=0.5, t_z=5.0, t_xy=15.0,
                    blocks=blocks, maxva=4.0e6, precision=precision)
    bg = fluxtube_background(nx, ny, nz, L, L, -25.0, 1.0)
    tab = psr_table(p, npulses, seed)
    src = psr_source(tab)
    return p, bg, src


# Grid spacing of the flux-tube configuration (256 points over 100 Mm,
# 300 points over -25..+1 Mm), kept by the ensemble members.
DX_MM = 100.0 / 256
DZ_MM = 26.0 / 299


def member_params(nx, nz, B0_gauss, precision=abi.SPARC_FP32,
                  blocks=(2, 2, 4)):
    """The run parameters of member() alone (no background arrays)."""
    L = nx * DX_MM * MM
    quiet = B0_gauss <= 0.0
    return base_params(nx, nx, nz, magnetic=0 if quiet else 2, periodic=quiet,
                       hpml=not quiet, xlength=L, ylength=L, timestep=0.5,
                       t_z=5.0, t_xy=15.0, blocks=blocks, maxva=4.0e6,
                       precision=precision)


def member(nx, nz, B0_gauss, depth_mm, precision=abi.SPARC_FP32,
           blocks=(2, 2, 4)):
    """One ensemble member: an nx x nx x nz box at the flux-tube spacing
    whose top is at +1 Mm.  B0 = 0: quiet (periodic, z-CPML, the hydro
    equations); B0 > 0: a flux tube (CPML on six faces, the MHD equations,
    Alfven speed capped at 40 km/s).  One PULSE = 1 Gaussian source at the
    horizontal centre at depth depth_mm; dt = 0.5 s, z filter every 10
    steps, xy filter every 30."""
    L = nx * DX_MM * MM
    z_bot = 1.0 - (nz - 1) * DZ_MM
    quiet = B0_gauss <= 0.0
    p = member_params(nx, nz, B0_gauss, precision, blocks)
    if quiet:
        bg = quiet_background(nx, nx, nz, z_bot, 1.0)
    else:
        bg = fluxtube_background(nx, nx, nz, L, L, z_bot, 1.0, B0=B0_gauss)
    src = pulse_source(px=0.5 * L, py=0.5 * L, pz=depth_mm * MM, t1=150.0,
                       st=40.0)
    return p, bg, src


def ensemble_draws(n=64, seed=SEED_CFG3):
    """The batched-ensemble members: nx = ny uniform in {96, 128, 160, 192,
    256}, nz uniform in [150, 300], B0 uniform in {0, 0.5, ..., 3} kG (the
    seeded B0 = 0 members are the quiet ones), source depth uniform in
    [-2, 0] Mm.  Returns a list of (nx, nz, B0_gauss, depth_mm)."""
    rng = np.random.Generator(np.random.Philox(key=seed))
    nxs = rng.choice([96, 128, 160, 192, 256], size=n)
    nzs = rng.integers(150, 301, size=n)
    b0 = 500.0 * rng.integers(0, 7, size=n)
    depth = -2.0 * rng.random(n)
    return [(int(a), int(b), float(c), float(d))
            for a, b, c, d in zip(nxs, nzs, b0, depth)]


def serve_draws(rate, duration_s, seed=SEED_CFG4, steps_scale=1.0):
    """Served-solve requests: Poisson arrivals at `rate` per second over
    duration_s seconds.  Each request draws nx = ny uniform in [64, 256], nz
    uniform in [128, 300], a background (quiet, or a flux tube with B0
    uniform in [0.5, 3] kG, even odds), a source (one Gaussian pulse, or a
    PULSE = 2 field of 50-500 pulses, even odds) and a duration of 500-4000
    driver iterations (times steps_scale, at least 20).  Returns a list of
    dicts sorted by arrival time."""
    rng = np.random.Generator(np.random.Philox(key=seed + int(rate * 1000)))
    out = []
    t = 0.0
    n = 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration_s:
            break
        tube = rng.random() < 0.5
        psr = rng.random() < 0.5
        out.append(dict(
            arrival=t, key=n,
            nx=int(rng.integers(64, 257)), nz=int(rng.integers(128, 301)),
            B0=float(rng.uniform(500.0, 3000.0)) if tube else 0.0,
            npulses=int(rng.integers(50, 501)) if psr else 0,
            depth=float(-2.0 * rng.random()),
            steps=max(20, int(round(rng.integers(500, 4001) * steps_scale))),
            seed=int(rng.integers(0, 2**62))))
        n += 1
    return out


def serve_request(d, precision=abi.SPARC_FP32, blocks=(2, 2, 4)):
    """(params, background, source) of a served request drawn by
    serve_draws: the ensemble member geometry and numerics, with the PULSE
    = 2 field when npulses > 0."""
    p, bg, src = member(d["nx"], d["nz"], d["B0"], d["depth"],
                        precision=precision, blocks=blocks)
    if d["npulses"] > 0:
        src = psr_source(psr_table(p, d["npulses"], d["seed"]))
    return p, bg, src
