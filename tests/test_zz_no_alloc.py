"""sparc_ke_norm_noalloc (the allocation-free reduction) against the
existing entry point that reports the same quantity, sparc_diagnostics'
ke_norm, on two calls in a row, through the C ABI.  Runs alone or after the
rest of the suite (it is collected last): the static scratch's counter is
reset by every call.

The two reductions sum the same per-point values in different orders:
agreement to 1e-12 relative.
"""
import ctypes as C

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
