"""The precision form (SPARC_FP32) against the FP64 plain form.

The FP64 plain form is itself pinned to the oracle at 1e-11 relative L2 per
field (test_gpu_parity.py), so it stands in for the FP64 oracle here; the
cfg0-sized test also compares with the oracle directly.

Tolerances: one iteration from a random state agrees to 1e-5 relative L2
per field (FP32 rounding of the stencils and RHS, ~1e-7 per operation); the
required bar for the precision form is 1e-4 relative L2 per field after
1000 steps.
"""
import numpy as np
import pytest

import oracle
from sparc2_b200 import Simulation, abi, workloads as W
from tests import cases
from tests.cases import rel_l2

pytestmark = pytest.mark.gpu

STEP_TOL32 = 1e-5
LONG_TOL32 = 1e-4

CASES32 = dict(cases.CASES)
# nx not a multiple of 4: the MHD kernel fetches own points by cp.async
CASES32["mhd_hpml_nx42"] = lambda: cases.mhd_hpml(nx=42, ny=40)


def twins(name):
    p, bg, src = CASES32[name]()
    s64 = Simulation(p, bg, src)
    p32, _, _ = CASES32[name]()
    p32.precision = abi.SPARC_FP32
    return s64, Simulation(p32, bg, src)


def max_norm(x, ref):
    d = np.max(np.abs(ref))
    return np.max(np.abs(x - ref)) / d if d > 0 else np.max(np.abs(x))


def test_state_round_trip():
    """set_state / get_state of the precision form: one FP32 rounding of the
    depth-scaled value."""
    _, s32 = twins("mhd_hpml")
    a0, psi0 = cases.random_state(s32, seed=4)
    s32.set_state(a0, psi0)
    a, psi = s32.get_state()
    assert np.max(np.abs(a - a0) / np.maximum(np.abs(a0), 1e-30)) < 3e-7
    assert np.max(np.abs(psi - psi0) / np.maximum(np.abs(psi0), 1e-30)) < 3e-7


@pytest.mark.parametrize("name", sorted(CASES32))
def test_one_iteration_fp32(name):
    s64, s32 = twins(name)
    a0, psi0 = cases.random_state(s64, seed=101)
    for s in (s64, s32):
        s.set_state(a0, psi0)
        s.step(3)
    ga, gpsi = s32.get_state()
    oa, opsi = s64.get_state()
    for l in range(s64.V):
        assert rel_l2(ga[l], oa[l]) <= STEP_TOL32, (l, rel_l2(ga[l], oa[l]))
    if s64.n_psi:
        assert rel_l2(gpsi, opsi) <= STEP_TOL32
    d32, _ = s32.diagnostics()
    d64, _ = s64.diagnostics()
    assert d32.iteration == d64.iteration == 3
    assert d32.ke_norm == pytest.approx(d64.ke_norm, rel=1e-5)
    assert d32.min_rho == pytest.approx(d64.min_rho, rel=1e-6)
    assert d32.min_p == pytest.approx(d64.min_p, rel=1e-6)


@pytest.mark.parametrize("name", ["quiet_periodic", "mhd_hpml"])
def test_filter_vars_fp32(name):
    s64, s32 = twins(name)
    a0, psi0 = cases.random_state(s64, seed=7)
    for s in (s64, s32):
        s.set_state(a0, psi0)
        s.filter_vars(30)
    ga, _ = s32.get_state()
    oa, _ = s64.get_state()
    for l in range(s64.V):
        assert rel_l2(ga[l], oa[l]) <= 1e-6, l


def test_filter_vars_7point_fp32():
    """filter_mode 2 on both axes in the precision form (the z pass's scale
    and the first pass's carry with the 7-point filter)."""
    ps = []
    for prec in (abi.SPARC_FP64, abi.SPARC_FP32):
        p, bg, src = cases.mhd_hpml(nz=80)
        p.filter_mode_xy = p.filter_mode_z = 2
        p.precision = prec
        ps.append(Simulation(p, bg, src))
    s64, s32 = ps
    a0, psi0 = cases.random_state(s64, seed=7)
    for s in (s64, s32):
        s.set_state(a0, psi0)
        s.step(3)
        s.filter_vars(30)
    ga, _ = s32.get_state()
    oa, _ = s64.get_state()
    for l in range(s64.V):
        assert rel_l2(ga[l], oa[l]) <= STEP_TOL32, l


@pytest.mark.parametrize("name", ["quiet_periodic", "mhd_hpml"])
def test_graph_run_equals_call_sequence_fp32(name):
    p, bg, src = CASES32[name]()
    p.precision = abi.SPARC_FP32
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


@pytest.mark.parametrize("name,steps", [("quiet_periodic", 300),
                                        ("quiet_hpml", 200),
                                        ("mhd_hpml", 200),
                                        ("mhd_hpml_nx42", 100),
                                        ("thermal_hpml", 120),
                                        ("mhd_periodic", 120),
                                        ("quiet_random", 120),
                                        ("mhd_random", 80)])
def test_many_iterations_fp32(name, steps):
    s64, s32 = twins(name)
    s64.run(0, steps)
    s32.run(0, steps)
    ga, gpsi = s32.get_state()
    oa, opsi = s64.get_state()
    for l in range(s64.V):
        e = rel_l2(ga[l], oa[l])
        assert e <= LONG_TOL32, (l, e)
    if s64.n_psi:
        assert rel_l2(gpsi, opsi) <= LONG_TOL32
    d32, r32 = s32.diagnostics()
    d64, r64 = s64.diagnostics()
    assert r32 == r64 == abi.SPARC_OK
    assert d32.ke_norm == pytest.approx(d64.ke_norm, rel=1e-4)


def test_cfg0_fp32_errors_at_100_500_1000():
    """Plain quiet-Sun hydro at full size in the precision form: relative L2
    and max-norm error per field against the FP64 oracle at iterations 100,
    500 and 1000, each within 1e-4 relative L2."""
    p, bg, src = W.cfg0()
    orc = oracle.Oracle(p, bg, src)
    p32, _, _ = W.cfg0(precision=abi.SPARC_FP32)
    s32 = Simulation(p32, bg, src)
    done = 0
    for mark in (100, 500, 1000):
        s32.run(done, mark + 1 - done)
        orc.run(done, mark + 1 - done)
        done = mark + 1
        ga, _ = s32.get_state()
        oa, _ = orc.get_state()
        errs = [rel_l2(ga[l], oa[l]) for l in range(s32.V)]
        mx = [max_norm(ga[l], oa[l]) for l in range(s32.V)]
        print(f"iteration {mark}: rel L2 {errs} max-norm {mx}")
        assert max(errs) <= LONG_TOL32, (mark, errs)
    assert np.max(np.abs(oa[3])) > 0


def test_cfg2_fp32_errors_at_100_500_1000():
    """The precision form on the flux-tube configuration at full size
    (256x256x300, 200 PSR pulses): relative L2 and max-norm error per field
    against the FP64 plain form (itself within 1e-11 of the oracle) at
    iterations 100, 500 and 1000, each within 1e-4 relative L2."""
    p64, bg, src = W.cfg1()
    s64 = Simulation(p64, bg, src)
    p32, _, _ = W.cfg1(precision=abi.SPARC_FP32)
    s32 = Simulation(p32, bg, src)
    del bg
    done = 0
    for mark in (100, 500, 1000):
        for s in (s64, s32):
            s.run(done, mark + 1 - done)
        done = mark + 1
        ga, _ = s32.get_state()
        oa, _ = s64.get_state()
        errs = [rel_l2(ga[l], oa[l]) for l in range(s32.V)]
        mx = [max_norm(ga[l], oa[l]) for l in range(s32.V)]
        print(f"cfg2 iteration {mark}: rel L2 {[f'{e:.2e}' for e in errs]} "
              f"max-norm {[f'{e:.2e}' for e in mx]}")
        assert max(errs) <= LONG_TOL32, (mark, errs)
        del ga, oa
    d32, r32 = s32.diagnostics()
    d64, r64 = s64.diagnostics()
    assert r32 == r64 == abi.SPARC_OK
    assert d32.ke_norm == pytest.approx(d64.ke_norm, rel=1e-4)
