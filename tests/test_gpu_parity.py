"""Parity of the CUDA path (through the C ABI) with the oracle.

Tolerances: the setup kernels are compiled without FMA contraction and
reproduce the oracle to a few ulp (1e-13 relative; exp/pow/sin may differ
by an ulp between CUDA and glibc).  The fused stage kernels contract to FMA,
so one step agrees to ~1e-14 relative L2 per field; the required bar for
the FP64 plain form is 1e-11 relative L2 per field after 1000 steps.
"""
import numpy as np
import pytest

import oracle
from sparc2_b200 import Simulation, abi, workloads as W
from tests import cases
from tests.cases import rel_l2

pytestmark = pytest.mark.gpu

STEP_TOL = 1e-12       # one driver iteration from a random state
LONG_TOL = 1e-11       # after many iterations (the FP64 plain-form bar)
COEF_TOL = 1e-13


def pair(name, **kw):
    p, bg, src = cases.CASES[name](**kw)
    return Simulation(p, bg, src), oracle.Oracle(p, bg, src)


@pytest.mark.parametrize("name", ["quiet_periodic", "mhd_hpml", "thermal_hpml"])
def test_setup_coefficients(name):
    sim, orc = pair(name)
    so, oo = sim.scalars(), orc.scalars()
    for k in so:
        assert so[k] == pytest.approx(oo[k], rel=1e-15, abs=0), k
    names = ["rho0", "p0", "rhoinv", "c2rho0", "gradrho0_z", "gradp0_z",
             "spongexyz", "source_damp", "stretch", "gblk", "a_z_bot",
             "b_z_bot", "kappa_z_top", "a_z_top"]
    if sim.params.magnetic == 2:
        names += ["reduction", "curlbox", "curlboy", "curlboz", "gradrho0_x",
                  "gradp0_y", "src_scale_beta", "box", "boz"]
    if sim.params.use_hpml:
        names += ["a_x_bot", "b_x_top", "kappa_y_bot", "b_y_top"]
    for n in names:
        g, o = sim.coeff(n), orc.coeff(n)
        assert g.shape == o.shape, n
        assert rel_l2(g, o) <= COEF_TOL, (n, rel_l2(g, o))


@pytest.mark.parametrize("name", ["quiet_periodic", "mhd_hpml"])
@pytest.mark.parametrize("dir", [0, 1, 2])
@pytest.mark.parametrize("bc", [1, 5])
def test_derivative_primitive(name, dir, bc):
    sim, orc = pair(name)
    rng = np.random.default_rng(3 + dir + 10 * bc)
    f = rng.standard_normal(sim.shape)
    g = sim.derivative(dir, bc, f)
    o = orc.derivative(dir, bc, f)
    assert np.max(np.abs(g - o)) <= 1e-13 * np.max(np.abs(o))


@pytest.mark.parametrize("name", ["quiet_periodic", "mhd_hpml"])
@pytest.mark.parametrize("dir", [0, 1, 2])
def test_filter_primitive(name, dir):
    sim, orc = pair(name)
    f = np.random.default_rng(7 + dir).standard_normal(sim.shape)
    g = sim.filter_field(dir, f)
    o = orc.filter_field(dir, f)
    assert np.max(np.abs(g - o)) <= 1e-14 * np.max(np.abs(o))


@pytest.mark.parametrize("name", sorted(cases.CASES))
def test_one_iteration_from_random_state(name):
    sim, orc = pair(name)
    a0, psi0 = cases.random_state(sim, seed=101)
    for s in (sim, orc):
        s.set_state(a0, psi0)
    nn = 3
    sim.step(nn)
    orc.step(nn)
    ga, gpsi = sim.get_state()
    oa, opsi = orc.get_state()
    for l in range(sim.V):
        assert rel_l2(ga[l], oa[l]) <= STEP_TOL, (l, rel_l2(ga[l], oa[l]))
    if sim.n_psi:
        assert rel_l2(gpsi, opsi) <= STEP_TOL
    gd, _ = sim.diagnostics()
    od, _ = orc.diagnostics()
    assert gd.iteration == od.iteration == nn
    assert gd.ke_norm == pytest.approx(od.ke_norm, rel=1e-12)
    assert gd.min_rho == pytest.approx(od.min_rho, rel=1e-13)
    assert gd.min_p == pytest.approx(od.min_p, rel=1e-13)


@pytest.mark.parametrize("name,kw", [("quiet_periodic", {}), ("mhd_hpml", {}), ("quiet_hpml", {}),
                                     ("quiet_hpml", {"nx": 41, "ny": 38})])
def test_filter_vars(name, kw):
    """The 11-point filter on both axes.  Grids with an even nx take the z
    pass whose slabs arrive as tensor copies, non-periodic ones also the xy
    pass with tensor-copied neighbourhoods; nx = 41 (rows not a multiple of
    16 bytes) takes the per-thread copies in both passes, the periodic grid
    in the xy pass."""
    sim, orc = pair(name, **kw)
    a0, psi0 = cases.random_state(sim, seed=7)
    for s in (sim, orc):
        s.set_state(a0, psi0)
    nn = 30  # a multiple of both cadences: xy and z pass
    sim.filter_vars(nn)
    orc.filter_vars(nn)
    ga, _ = sim.get_state()
    oa, _ = orc.get_state()
    for l in range(sim.V):
        assert rel_l2(ga[l], oa[l]) <= 1e-14, l


@pytest.mark.parametrize("name,kw", [("quiet_periodic", {}), ("mhd_hpml", {"nz": 80}),
                                     ("quiet_hpml", {"nx": 70, "ny": 66}),
                                     ("quiet_hpml", {"nx": 41, "ny": 38})])
def test_filter_vars_7point(name, kw):
    """filter_mode 2 on both axes (derivatives.f90: the 7-point filter,
    combined as a - s*filt, zero at the x/y edge points): nz = 80 gives the
    z pass slabs away from both ends and slabs at them; 70 x 66 gives xy
    tiles with and without the edge pre-average; nx = 41 the per-thread
    copies on a non-periodic grid."""
    p, bg, src = cases.CASES[name](**kw)
    p.filter_mode_xy = p.filter_mode_z = 2
    sim, orc = Simulation(p, bg, src), oracle.Oracle(p, bg, src)
    a0, psi0 = cases.random_state(sim, seed=8)
    for s in (sim, orc):
        s.set_state(a0, psi0)
    sim.filter_vars(30)
    orc.filter_vars(30)
    ga, _ = sim.get_state()
    oa, _ = orc.get_state()
    for l in range(sim.V):
        assert rel_l2(ga[l], oa[l]) <= 1e-14, l


@pytest.mark.parametrize("name", ["quiet_periodic", "mhd_hpml"])
def test_graph_run_equals_call_sequence(name):
    """sparc_run (CUDA graphs) == sparc_step + sparc_filter_vars, bitwise."""
    p, bg, src = cases.CASES[name]()
    s1, s2 = Simulation(p, bg, src), Simulation(p, bg, src)
    a0, psi0 = cases.random_state(s1, seed=9, amp=1e-6)
    s1.set_state(a0, psi0)
    s2.set_state(a0, psi0)
    s1.run(0, 35)
    for nn in range(35):
        s2.step(nn)
        s2.filter_vars(nn)
    a1, p1 = s1.get_state()
    a2, p2 = s2.get_state()
    assert np.array_equal(a1, a2)
    assert np.array_equal(p1, p2)
    d1, _ = s1.diagnostics()
    d2, _ = s2.diagnostics()
    assert d1.ke_norm == d2.ke_norm and d1.iteration == d2.iteration == 34


@pytest.mark.parametrize("name,steps", [("quiet_periodic", 300),
                                        ("mhd_hpml", 200),
                                        ("thermal_hpml", 120),
                                        ("mhd_periodic", 120),
                                        ("mhd_hpml_96", 40),
                                        ("quiet_random", 120),
                                        ("mhd_random", 60)])
def test_many_iterations_from_rest(name, steps):
    """Driver loop from rest with the configured source, filters at cadence."""
    sim, orc = pair(name)
    sim.run(0, steps)
    orc.run(0, steps)
    ga, gpsi = sim.get_state()
    oa, opsi = orc.get_state()
    for l in range(sim.V):
        e = rel_l2(ga[l], oa[l])
        assert e <= LONG_TOL, (l, e)
    if sim.n_psi:
        assert rel_l2(gpsi, opsi) <= LONG_TOL
    gd, gr = sim.diagnostics()
    od, orr = orc.diagnostics()
    assert gr == orr == abi.SPARC_OK
    assert gd.ke_norm == pytest.approx(od.ke_norm, rel=1e-10)


def test_cfg0_1000_iterations():
    """Plain quiet-Sun hydro at its full size (64x64x128) for 1000 steps:
    the FP64 plain form within 1e-11 relative L2 per field."""
    p, bg, src = W.cfg0()
    sim = Simulation(p, bg, src)
    orc = oracle.Oracle(p, bg, src)
    sim.run(0, 1001)
    orc.run(0, 1001)
    ga, gpsi = sim.get_state()
    oa, opsi = orc.get_state()
    errs = [rel_l2(ga[l], oa[l]) for l in range(sim.V)]
    assert max(errs) <= LONG_TOL, errs
    assert rel_l2(gpsi, opsi) <= LONG_TOL
    assert np.max(np.abs(oa[3])) > 0  # the pulse did drive the box


def test_unstable_state_is_reported():
    """The fail criterion of driver.f90:175-183, triggered from the host by
    a non-physical state (negative total density)."""
    p, bg, src = cases.quiet_periodic()
    sim = Simulation(p, bg, src)
    a, psi = sim.get_state()
    a[0, 20, 10, 10] = -1.0e3          # rho + rho0 < 0 in the interior
    sim.set_state(a, psi)
    sim.step(5)
    d, r = sim.diagnostics()
    assert r == abi.SPARC_ERR_UNSTABLE
    assert d.fail_iteration == 5 and d.min_rho < 0
    # the handle stays usable; a healthy state reports no new failure index
    sim.step(6)
    d2, r2 = sim.diagnostics()
    assert d2.fail_iteration == 5 and d2.iteration == 6


def test_errors_cross_the_abi():
    p, bg, src = cases.quiet_periodic()
    p.block_z = 1
    with pytest.raises(abi.SparcError) as e:
        Simulation(p, bg, src)
    assert e.value.code == abi.SPARC_ERR_INVALID
    p, bg, src = cases.quiet_periodic()
    sim = Simulation(p, bg, src)
    bad = abi.SparcSource()
    bad.kind = abi.SPARC_SRC_PULSE
    bad.dir = 7
    with pytest.raises(abi.SparcError):
        sim.set_source(bad)


@pytest.mark.parametrize("precision", [abi.SPARC_FP64, abi.SPARC_FP32])
def test_set_source_again_replaces_the_source(precision):
    """A later sparc_set_source replaces an earlier one (the earlier tables
    are freed): after PSR, random, then PSR again the run is bitwise the run
    of a handle that only ever had the PSR source."""
    p, bg, psr = cases.mhd_hpml()
    _, _, rnd = cases.mhd_random(nx=p.nx, ny=p.ny, nz=p.nz)
    p.precision = precision
    a = Simulation(p, bg, psr)
    a.set_source(rnd)
    a.set_source(psr)
    b = Simulation(p, bg, psr)
    for s in (a, b):
        s.run(0, 12)
    ga, gpsi = a.get_state()
    ba, bpsi = b.get_state()
    assert np.array_equal(ga, ba) and np.array_equal(gpsi, bpsi)
    assert a.diagnostics()[0].ke_norm == b.diagnostics()[0].ke_norm
    a.close()
    b.close()


@pytest.mark.parametrize("name,kw", [("quiet_periodic", {}), ("quiet_hpml", {}),
                                     ("mhd_hpml", {"nx": 42, "nz": 64})])
def test_damping_against_the_oracle(name, kw):
    """DAMPING = 1: the FFT horizontal damping of the velocities in every
    RHS evaluation (cuFFT on the device, direct sums in the oracle), 12
    driver iterations through the CUDA-graph loop."""
    p, bg, src = cases.CASES[name](**kw)
    p.damping = 1
    sim, orc = Simulation(p, bg, src), oracle.Oracle(p, bg, src)
    a0, psi0 = cases.random_state(sim, seed=31)
    for s in (sim, orc):
        s.set_state(a0, psi0)
    sim.run(0, 12)
    orc.run(0, 12)
    ga, gpsi = sim.get_state()
    oa, opsi = orc.get_state()
    for l in range(sim.V):
        assert rel_l2(ga[l], oa[l]) <= 1e-11, (l, rel_l2(ga[l], oa[l]))
    if sim.n_psi:
        assert rel_l2(gpsi, opsi) <= 1e-11
    gd, _ = sim.diagnostics()
    od, _ = orc.diagnostics()
    assert gd.ke_norm == pytest.approx(od.ke_norm, rel=1e-11)


def test_damping_changes_the_velocities_only_through_the_term():
    """With and without DAMPING from the same state, one iteration: density
    and pressure of stage 1 see the damped velocities only from stage 2 on,
    and the damped run differs."""
    p, bg, src = cases.quiet_hpml()
    p2, _, _ = cases.quiet_hpml()
    p2.damping = 1
    s0, s1 = Simulation(p, bg, src), Simulation(p2, bg, src)
    a0, psi0 = cases.random_state(s0, seed=5)
    for s in (s0, s1):
        s.set_state(a0, psi0)
        s.step(3)
    a, _ = s0.get_state()
    b, _ = s1.get_state()
    assert not np.array_equal(a[1], b[1])
    # FP32 precision form: refused
    p3, _, _ = cases.quiet_hpml()
    p3.damping = 1
    p3.precision = abi.SPARC_FP32
    with pytest.raises(abi.SparcError):
        Simulation(p3, bg, src)
