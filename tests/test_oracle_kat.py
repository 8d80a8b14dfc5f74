"""Known-answer tests that pin the oracle (CPU only).

The reference ships no tests, golden vectors or fixtures, so these pin the
restatement analytically: stencil accuracy, filter transfer function, the
RK amplification polynomial, CPML profiles and rest-state invariance.
"""
import numpy as np
import pytest

import oracle
from sparc2_b200 import workloads as W
from tests import cases

# initialize.f90:1959-1969 centred row and 1366-1381 RK coefficients
C6 = np.array([-0.002484594688, 0.020779405824, -0.090320001280,
               0.286511173973, -0.872756993962, 0.0, 0.872756993962,
               -0.286511173973, 0.090320001280, -0.020779405824,
               0.002484594688])
GAMMA = [1.0, 0.5, 0.1665579725791151184, 0.03950410250586729987,
         0.007810706393337838236]


@pytest.fixture(scope="module")
def quiet():
    p, bg, src = cases.quiet_periodic()
    return oracle.Oracle(p, bg, src), p


def test_centred_stencil_is_antisymmetric():
    assert np.array_equal(C6, -C6[::-1])
    assert C6[5] == 0.0


@pytest.mark.parametrize("dir", [0, 1])
@pytest.mark.parametrize("kmode", [1, 3, 7])
def test_periodic_derivative_modified_wavenumber(quiet, dir, kmode):
    """ddx of sin(2 pi k x) on the periodic grid equals the Bogey-Bailly
    modified wavenumber times cos(...) (derivatives.f90:41)."""
    o, p = quiet
    n = p.nx if dir == 0 else p.ny
    q = np.arange(n) / n
    phase = 2 * np.pi * kmode * q
    f = np.sin(phase)
    field = np.broadcast_to(f[None, None, :] if dir == 0 else f[None, :, None],
                            o.shape).copy()
    d = o.derivative(dir, 5, field)
    stretch = o.scalars()["stretchx" if dir == 0 else "stretchy"]
    h = 2 * np.pi * kmode / n
    kmod = sum(2 * C6[5 + m] * np.sin(m * h) for m in range(1, 6))
    expect = stretch * kmod * np.cos(phase)
    got = d[3, 2, :] if dir == 0 else d[3, :, 2]
    assert np.max(np.abs(got - expect)) <= 1e-12 * stretch


def test_one_sided_rows_differentiate_linear_profiles(quiet):
    """One-sided rows 1-5 (initialize.f90:1971-2029) are first-order exact to
    the accuracy of the reference's hand perturbations; z uses them at the
    top (derivatives.f90:536-545)."""
    o, p = quiet
    z = o.coeff("zaxis")
    field = np.broadcast_to(z[:, None, None], o.shape).copy()
    d = o.derivative(2, 1, field)[:, 4, 4]
    assert np.max(np.abs(d[-5:] - 1.0)) < 1e-9
    assert np.max(np.abs(d[5:-5] - 1.0)) < 1e-12
    const = np.ones(o.shape)
    dc = o.derivative(2, 1, const)[:, 1, 1]
    stretch = o.coeff("stretch")
    assert np.max(np.abs(dc[-5:] / stretch[-5:])) < 1e-10
    assert np.max(np.abs(dc[5:-5] / stretch[5:-5])) < 1e-16


def test_filter_passes_constants_and_transfer_at_nyquist(quiet):
    o, p = quiet
    const = np.full(o.shape, 2.5)
    for d in range(3):
        assert np.allclose(o.filter_field(d, const), 2.5, rtol=0, atol=1e-15)
    # 11-point filter at the Nyquist mode: sum_m c_m (-1)^m
    c11 = np.array([0.5 * 0.001953125, -0.5 * 0.01953125, 0.5 * 0.087890625,
                    -0.5 * 0.234375, 0.5 * 0.41015625, 0.75390625,
                    0.5 * 0.41015625, -0.5 * 0.234375, 0.5 * 0.087890625,
                    -0.5 * 0.01953125, 0.5 * 0.001953125])
    nyq = (-1.0) ** np.arange(p.nx)
    field = np.broadcast_to(nyq[None, None, :], o.shape).copy()
    out = o.filter_field(0, field)[5, 5, :]
    gain = np.sum(c11 * (-1.0) ** np.arange(11))
    assert np.allclose(out, gain * nyq, atol=1e-15)
    assert abs(gain) < 1e-15


def test_rk_betas_give_the_amplification_polynomial(quiet):
    """step.f90:26-61 applied to F(u) = lambda u gives 1 + sum gamma_j z^j
    with the optimized gammas of initialize.f90:1368-1372."""
    o, _ = quiet
    s = o.scalars()
    dt = s["deltat"]
    b = [s[f"beta{k}"] / dt for k in range(1, 6)]
    # u1 = 1 + b5 z (1 + b4 z (1 + b3 z (1 + b2 z))) expanded
    g2 = b[4]
    g3 = b[4] * b[3]
    g4 = b[4] * b[3] * b[2]
    g5 = b[4] * b[3] * b[2] * b[1]
    assert b[0] == 0.0
    assert np.allclose([g2, g3, g4, g5], GAMMA[1:], rtol=1e-15)


def test_cpml_profiles_follow_initialize_f90():
    p, bg, src = cases.mhd_hpml()
    o = oracle.Oracle(p, bg, src)
    z = o.coeff("zaxis")
    npb = p.npml_zb
    L = z[npb - 1] - z[0]
    s = o.scalars()
    f0 = 3.14159265358979 * 0.005 * s["diml"] / s["dimc"]
    ratio = (z[npb - 1] - z[:npb]) / L
    kap = 1.0 + (p.pml_zb[2] - 1.0) * ratio ** p.pml_zb[1]
    got_k = o.coeff("kappa_z_bot").reshape(npb, p.ny, p.nx)
    assert np.allclose(got_k[:, 7, 9], kap, rtol=1e-15)
    alpha = f0 * (z[:npb] - z[0]) / L
    # b = -alpha - d/kappa and a = -d/kappa^2, so -(b + alpha) = -a*kappa
    a = o.coeff("a_z_bot").reshape(npb, p.ny, p.nx)
    b = o.coeff("b_z_bot").reshape(npb, p.ny, p.nx)
    assert np.allclose(-(b + alpha[:, None, None]), -a * kap[:, None, None],
                       rtol=1e-12, atol=1e-300)
    assert np.all(a[-1] == 0.0) and np.all(a[:-1] < 0.0)


@pytest.mark.parametrize("name", ["quiet_periodic", "mhd_hpml"])
def test_rest_state_without_source_stays_at_rest(name):
    p, bg, _ = cases.CASES[name]()
    o = oracle.Oracle(p, bg, None)
    o.run(0, 31)
    a, psi = o.get_state()
    assert np.all(a == 0.0) and np.all(psi == 0.0)


def test_psr_first_iteration_doubles_the_forcing():
    """all_modules.f90:592-611 then 614-660: at the run's first iteration
    every pulse is added twice."""
    p, bg, src = cases.mhd_hpml()
    o = oracle.Oracle(p, bg, src)
    f0 = o.forcing(0)
    src.init = 1
    o.set_source(src)
    f0b = o.forcing(0)
    assert np.allclose(f0, 2.0 * f0b, rtol=1e-14, atol=0)


def test_stabilise_clamp(quiet):
    """gradp0_z >= -rho0 g below the surface band (initialize.f90:1026)."""
    o, p = quiet
    gp = o.coeff("gradp0_z").reshape(o.shape)[:, 0, 0]
    rho0 = o.coeff("rho0").reshape(o.shape)[:, 0, 0]
    g = o.coeff("g")
    z = o.coeff("zaxis")
    sel = (z <= np.float32(0.9998)) & (np.arange(len(z)) >= p.npml_zb) & \
        (np.arange(len(z)) < len(z) - p.npml_zt)
    assert np.all(gp[sel] >= -rho0[sel] * g[sel] - 1e-300)


# ------------------------------------------------ PULSE = 0 random source
def _lagrange_point(vr, nn, dt, cad, ns):
    """LAGRANGE_INTERP (all_modules.f90:1892-1950) for one column's series
    vr[m] (0-based samples), the reference's operation order."""
    xt = nn * dt / cad
    time1 = int(np.floor(xt)) + 1
    xt = nn * dt
    x = [(time1 - 4 + j) * cad for j in range(7)]
    use = [x[j] >= 0 for j in range(4)] + [True, time1 < ns, time1 < ns - 1]
    f = 0.0
    for j in range(7):
        m = time1 - 4 + j
        lc = 0.0
        if use[j] and 0 <= m < ns:
            den = None
            for q in range(7):
                if q != j:
                    den = x[j] - x[q] if den is None else den * (x[j] - x[q])
            lc = vr[m] / den
        t = lc
        for q in range(7):
            if q != j:
                t = t * (xt - x[q])
        f = t if j == 0 else f + t
    return f


def _random_case(series_fn, nn_list, cad=10.0):
    p, bg, _ = cases.quiet_hpml(nx=24, ny=22, nz=24)
    ns = 2 * ((int(np.floor(400 * p.timestep / cad)) + 2) // 2) + 2
    tm = np.arange(ns) * cad
    series = series_fn(tm)[:, None, None] * (1.0 + 0.1 * np.arange(p.nx))[None, None, :] * \
        np.ones((1, p.ny, 1))
    src = W.random_source(series, cadforcing=cad, ampl=2.0e3, depth=-0.6 * W.MM,
                          sigma=0.4 * W.MM)
    o = oracle.Oracle(p, bg, src)
    dimc = o.scalars()["dimc"]
    out = [o.forcing(nn) for nn in nn_list]
    sd = o.coeff("source_damp").reshape(p.nz, p.ny, p.nx)[0]
    dep = o.coeff("source_dep")
    # e_rad and source_dep as all_modules.f90:289-301 state them
    z = o.coeff("zaxis")
    temp2, temp, e_rad = 1.0 + (-0.6 * W.MM) / W.RSUN, 1.0, 0
    for k in range(p.nz):
        if abs(z[k] - temp2) <= temp:
            temp, e_rad = abs(z[k] - temp2), k
    sg = 0.4 * W.MM / W.RSUN
    want = np.exp(-0.5 * (z - z[e_rad]) ** 2 / 2.0 / sg ** 2)
    assert np.array_equal(dep, want)
    return p, series, dimc, sd, dep, out, ns


def test_random_source_follows_the_reference_formula():
    """Early iterations drop the samples before t = 0 (x_j < 0), late ones
    those past the series; every value follows LAGRANGE_INTERP, times
    source_damp(:,:,1) and source_dep(k) (driver.f90:131-132, RHS.f90:147)."""
    nn_list = [0, 1, 7, 25, 41, 399]
    p, series, dimc, sd, dep, out, ns = _random_case(
        lambda t: np.sin(t / 37.0) + 0.2 * np.cos(t / 11.0), nn_list)
    vr = (2.0e3 / dimc) * series
    for nn, f in zip(nn_list, out):
        for (j, i) in [(0, 0), (3, 7), (21, 23)]:
            g = _lagrange_point(vr[:, j, i], nn, p.timestep, 10.0, ns) * sd[j, i]
            assert np.allclose(f[:, j, i], g * dep, rtol=1e-14, atol=0.0), (nn, j, i)
    assert dep.max() == 1.0 and dep.min() > 0.0


def test_random_source_reproduces_a_cubic_in_time():
    """With all seven samples in range, 7-point Lagrange interpolation is
    exact on a cubic in time (KAT of the restatement)."""
    T = 200.0
    P = lambda t: 1.0 + 0.3 * (t / T) - 0.2 * (t / T) ** 2 + 0.05 * (t / T) ** 3
    nn_list = [90, 133, 250]          # time1 in [4, ns - 2]
    p, series, dimc, sd, dep, out, ns = _random_case(P, nn_list)
    for nn, f in zip(nn_list, out):
        t = nn * p.timestep
        want = (2.0e3 / dimc) * P(t) * (1.0 + 0.1 * np.arange(p.nx))[None, :] * sd
        got = f / dep[:, None, None]
        assert np.allclose(got, want[None], rtol=1e-11, atol=0.0), nn
