"""z extent of the stage kernels' work items (sparc_set_zchunk, sparc_tune):
the chunking changes only which CTA computes a layer (each chunk warms its
own z windows from the same values), so the state is bitwise the same for
every extent, and the autotuner's trial iterations are real iterations of
the driver loop."""
import numpy as np
import pytest

from sparc2_b200 import Simulation, abi
from tests import cases

pytestmark = pytest.mark.gpu

PRECS = [abi.SPARC_FP64, abi.SPARC_FP32]


def sim_of(name, prec, **kw):
    p, bg, src = cases.CASES[name](**kw)
    p.precision = prec
    return Simulation(p, bg, src)


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("name", ["mhd_hpml", "quiet_hpml"])
def test_extent_does_not_change_results(name, prec):
    res = []
    for zc in (None, 11, 16, 29, 200):
        s = sim_of(name, prec, nz=72)
        if zc is not None:
            s.set_zchunk(zc)
            assert s.zchunk == min(zc, 72)
        s.run(0, 31)
        res.append(s.get_state())
        s.close()
    for a, psi in res[1:]:
        assert np.array_equal(a, res[0][0])
        assert np.array_equal(psi, res[0][1])


@pytest.mark.parametrize("prec", PRECS)
def test_tuner_runs_real_iterations(prec):
    ref = sim_of("mhd_hpml", prec, nz=72)
    s = sim_of("mhd_hpml", prec, nz=72)
    nxt, best = s.tune(0, steps_per_trial=1)
    assert 11 <= best <= 72 and s.zchunk == best
    assert nxt > 5
    s.run(nxt, 40 - nxt)
    ref.run(0, 40)
    a, psi = s.get_state()
    ra, rpsi = ref.get_state()
    assert np.array_equal(a, ra) and np.array_equal(psi, rpsi)
    d, _ = s.diagnostics()
    rd, _ = ref.diagnostics()
    assert d.iteration == rd.iteration == 39
    assert d.ke_norm == rd.ke_norm


def test_extent_limits():
    s = sim_of("quiet_periodic", abi.SPARC_FP64)
    with pytest.raises(abi.SparcError):
        s.set_zchunk(10)
    with pytest.raises(abi.SparcError):
        s.tune(0, steps_per_trial=0)
