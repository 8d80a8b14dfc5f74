"""Failure detection without a GPU fault: a bounded device wait that runs
out (an mbarrier that nothing completes) raises the handle's error flag;
the host reads SPARC_ERR_TIMEOUT, the context stays usable, and a restart
from saved state clears the flag and steps on as if nothing happened."""
import numpy as np
import pytest

from sparc2_b200 import Simulation, abi
from tests import cases

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [abi.SPARC_FP64, abi.SPARC_FP32])
def test_gave_up_wait_is_reported_and_cleared_by_a_restart(precision):
    p, bg, src = cases.quiet_periodic()
    p.precision = precision
    sim = Simulation(p, bg, src)
    ref = Simulation(p, bg, src)
    for s in (sim, ref):
        s.run(0, 6)
    a, psi = sim.get_state()
    assert sim.lib.sparc_inject_wait_timeout(sim.h, 200) == abi.SPARC_OK
    with pytest.raises(abi.SparcError) as e:
        sim.diagnostics()
    assert e.value.code == abi.SPARC_ERR_TIMEOUT
    assert sim.lib.sparc_inject_wait_timeout(sim.h, 0) == abi.SPARC_ERR_INVALID
    assert sim.lib.sparc_inject_wait_timeout(sim.h, (1 << 20) + 1) == abi.SPARC_ERR_INVALID
    sim.set_state(a, psi)          # restart from the saved state
    d, r = sim.diagnostics()
    assert r == abi.SPARC_OK
    for s in (sim, ref):
        s.run(6, 6)
    ga, _ = sim.get_state()
    ra, _ = ref.get_state()
    if precision == abi.SPARC_FP64:
        assert np.array_equal(ga, ra)
    else:   # the restart re-rounds the depth-scaled FP32 state once
        assert max(cases.rel_l2(ga[l], ra[l]) for l in range(sim.V)) < 1e-5
    assert sim.diagnostics()[0].iteration == ref.diagnostics()[0].iteration == 11
    sim.close()
    ref.close()
