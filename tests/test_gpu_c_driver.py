"""The C caller of the ABI (sparc2_b200/host/sparc_driver.c, the driver.f90
loop: step, diagnostics, filter) on the device, with pulse, PULSE = 2 and
PULSE = 0 sources: its per-iteration diagnostics equal those of the Python
host loop over the same library calls, bit for bit."""
import pytest

from sparc2_b200 import Simulation
from tests import c_driver, cases

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["quiet_periodic", "mhd_periodic", "mhd_hpml", "quiet_random"])
def test_c_driver_matches_the_python_loop(tmp_path, name):
    exe = c_driver.build(tmp_path)
    p, bg, src = cases.CASES[name]()
    c_driver.write_inputs(tmp_path, p, bg, src)
    r = c_driver.run(exe, tmp_path, 0, 35)
    assert r.returncode == 0, r.stderr
    rows = [line.split() for line in r.stdout.strip().splitlines()]
    assert len(rows) == 35
    sim = Simulation(p, bg, src)
    for nn in range(35):
        sim.step(nn)
        d, st = sim.diagnostics()
        got = rows[nn]
        assert int(got[0]) == nn and int(got[4]) == st
        assert float(got[1]) == d.ke_norm and float(got[2]) == d.min_rho
        assert float(got[3]) == d.min_p
        if nn:
            sim.filter_vars(nn)
    sim.close()


@pytest.mark.parametrize("name", ["quiet_periodic", "mhd_hpml"])
def test_c_driver_from_a_trol_file(tmp_path, name):
    """The C caller started from a .trol file runs the same iterations as
    the Python loop over the parameters sparc_parse_trol reads from it."""
    import ctypes as C
    from sparc2_b200 import abi
    exe = c_driver.build(tmp_path)
    p, bg, src = cases.CASES[name]()
    c_driver.write_inputs(tmp_path, p, bg, src)
    text = c_driver.trol_text(p, src)
    (tmp_path / "run.trol").write_text(text)
    r = c_driver.run(exe, tmp_path, 0, 25, "--trol", str(tmp_path / "run.trol"))
    assert r.returncode == 0, r.stderr
    rows = [line.split() for line in r.stdout.strip().splitlines()]
    t = abi.SparcTrol()
    lib = abi.load()
    assert lib.sparc_parse_trol(text.encode(), C.byref(t), None, 0) == abi.SPARC_OK
    tp = t.params
    if src.kind == abi.SPARC_SRC_PSR:
        s2 = src
    else:
        s2 = t.source
    sim = Simulation(tp, bg, s2)
    for nn in range(25):
        sim.step(nn)
        d, st = sim.diagnostics()
        got = rows[nn]
        assert int(got[0]) == nn and int(got[4]) == st
        assert float(got[1]) == d.ke_norm and float(got[2]) == d.min_rho
        if nn:
            sim.filter_vars(nn)
    sim.close()
