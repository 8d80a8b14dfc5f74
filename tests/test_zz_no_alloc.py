"""sparc_ke_norm_noalloc (the allocation-free reduction) against the
existing entry point that reports the same quantity, sparc_diagnostics'
ke_norm, on two calls in a row, through the C ABI.  Runs alone or after the
rest of the suite (it is collected last): the static scratch's counter is
reset by every call.

The two reductions sum the same per-point values in different orders:
agreement to 1e-12 relative.
"""
import ctypes as C

import numpy as np
import pytest

from sparc2_b200 import Simulation, abi
from sparc2_b200 import workloads as W
from tests import cases

pytestmark = pytest.mark.gpu


def noalloc(sim):
    out = C.c_double()
    r = sim.lib.sparc_ke_norm_noalloc(sim.h, C.byref(out))
    return r, out.value


@pytest.mark.parametrize("name,precision", [("quiet_periodic", abi.SPARC_FP64),
                                            ("mhd_hpml", abi.SPARC_FP64),
                                            ("mhd_hpml", abi.SPARC_FP32),
                                            ("quiet_periodic", abi.SPARC_FP32)])
def test_matches_diagnostics_two_calls_in_a_row(name, precision):
    p, bg, src = cases.CASES[name]()
    p.precision = precision
    sim = Simulation(p, bg, src)
    sim.run(0, 40)                    # from rest, driven by the source
    for nn in (40, 41):
        sim.step(nn)
        d, r = sim.diagnostics()
        assert r == abi.SPARC_OK
        rn, ke = noalloc(sim)
        assert rn == abi.SPARC_OK, sim.lib.sparc_last_error(sim.h)
        assert d.ke_norm > 0
        assert ke == pytest.approx(d.ke_norm, rel=1e-12), (nn, ke, d.ke_norm)


def test_batch_members_read_their_live_state():
    """In a batch the buffer roles rotate on the device every step; the
    entry point must reduce each member's live state, before and after the
    members leave the batch."""
    from sparc2_b200.batch import Batch
    sims = []
    for name in ("mhd_hpml", "quiet_periodic"):
        p, bg, src = cases.CASES[name]()
        p.precision = abi.SPARC_FP32
        sims.append(Simulation(p, bg, src))
    with Batch(4) as b:
        slots = [b.add(s, 0, 7) for s in sims]
        # seven iterations 0..6 (no filter cadence): diagnostics' ke_norm
        # is the norm of the state the batch left in role 0
        b.run(7)
        b.synchronize()
        for s in sims:
            d, r = s.diagnostics()
            assert r == abi.SPARC_OK and d.ke_norm > 0
            rn, ke = noalloc(s)
            assert rn == abi.SPARC_OK, s.lib.sparc_last_error(s.h)
            assert ke == pytest.approx(d.ke_norm, rel=1e-12), (ke, d.ke_norm)
        for q in slots:
            b.remove(q)
    for s in sims:
        d, _ = s.diagnostics()
        rn, ke = noalloc(s)
        assert rn == abi.SPARC_OK
        assert ke == pytest.approx(d.ke_norm, rel=1e-12)


def test_norm_is_of_the_current_state_after_a_filter():
    """After FILTER_VARS the state differs from the stage-5 state whose norm
    sparc_diagnostics keeps; the entry point reduces the current state."""
    p, bg, src = cases.CASES["quiet_periodic"]()
    sim = Simulation(p, bg, src)
    sim.run(0, 29)
    sim.step(29)
    sim.filter_vars(29)               # 29 is not a cadence: no change
    d, _ = sim.diagnostics()
    assert noalloc(sim)[1] == pytest.approx(d.ke_norm, rel=1e-12)
    sim.step(30)
    sim.filter_vars(30)               # xy and z filters at iteration 30
    d, _ = sim.diagnostics()
    a, _ = sim.get_state()
    sc = sim.scalars()
    rho0 = sim.coeff("rho0")
    rho0 = rho0.reshape(a.shape[1:]) if rho0.size == a[0].size else rho0[:, None, None]
    m = (rho0 + a[0]) * (a[1] ** 2 + a[2] ** 2 + a[3] ** 2) / 2.0
    want = np.sqrt(np.sum(m * m) / m.size) * sc["dimc"] ** 2 * sc["dimrho"]
    got = noalloc(sim)[1]
    assert got == pytest.approx(want, rel=1e-12)
    assert got != pytest.approx(d.ke_norm, rel=1e-9)


def test_grid_above_the_scratch_limit_is_rejected():
    p, _, _ = W.cfg0(nx=512, ny=512, nz=257, precision=abi.SPARC_FP32)
    h = C.c_void_p()
    lib = abi.load()
    assert lib.sparc_create(C.byref(p), 0, C.byref(h)) == abi.SPARC_OK
    out = C.c_double()
    try:
        assert lib.sparc_ke_norm_noalloc(h, C.byref(out)) == abi.SPARC_ERR_INVALID
        assert b"67108864-point limit" in lib.sparc_last_error(h)
    finally:
        lib.sparc_destroy(h)
