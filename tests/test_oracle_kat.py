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
