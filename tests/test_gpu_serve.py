"""The serving loop: requests that arrive while others run are admitted by
memory budget and slots, overlap on the device, and each result is the same
as the request run alone (FP32-level tolerance, 1e-6 relative L2 per field:
the batched kernels evaluate the same per-point arithmetic on other tile
shapes)."""
import numpy as np
import pytest

from sparc2_b200 import Simulation, abi
from sparc2_b200.serve import Server, drive, estimate_bytes
from tests import cases
from tests.cases import rel_l2

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(300)]

KINDS = {
    "quiet_periodic": cases.quiet_periodic,
    "quiet_hpml": cases.quiet_hpml,
    "thermal_hpml": cases.thermal_hpml,
    "mhd_hpml": cases.mhd_hpml,
    "mhd_periodic": cases.mhd_periodic,
}


def fp32(kind):
    p, bg, src = KINDS[kind]()
    p.precision = abi.SPARC_FP32
    return p, bg, src


def alone(kind, steps):
    s = Simulation(*fp32(kind))
    s.run(0, steps)
    a, psi = s.get_state()
    d, _ = s.diagnostics()
    s.close()
    return a, psi, d


def test_served_results_equal_their_alone_runs():
    plan = [(0.00, "mhd_hpml", 45), (0.02, "quiet_periodic", 30),
            (0.05, "thermal_hpml", 25), (0.08, "mhd_periodic", 35),
            (0.10, "quiet_hpml", 20), (0.12, "mhd_hpml", 15)]
    requests = []
    for key, (arr, kind, steps) in enumerate(plan):
        p, _, _ = fp32(kind)
        requests.append((arr, key, p, 0, steps))
    got = {}

    def build(key):
        _, bg, src = fp32(plan[key][1])
        return bg, src

    def on_result(key, sim, state, times):
        assert state == abi.SPARC_REQ_DONE
        a, psi = sim.get_state()
        d, _ = sim.diagnostics()
        got[key] = (a, psi, d, times)

    with Server(capacity=3, budget_bytes=8 << 30, quantum=4) as srv:
        drive(srv, requests, build, on_result, deadline_s=200)
        st = srv.stats()
    assert len(got) == len(plan)
    assert st["max_concurrent"] <= 3
    # continuous batching: requests ran on the device together, and some
    # joined a batch that was already running others
    assert st["max_running"] >= 2, st
    assert st["joined_running"] >= 1, st
    spans = [got[k][3][2:4] for k in got]        # (start, done) per request
    overlap = [(a, b) for a in range(len(spans)) for b in range(a + 1, len(spans))
               if spans[a][0] < spans[b][1] and spans[b][0] < spans[a][1]]
    assert overlap, spans
    for key, (arr, kind, steps) in enumerate(plan):
        a, psi, d, times = got[key]
        ra, rpsi, rd = alone(kind, steps)
        for l in range(a.shape[0]):
            assert rel_l2(a[l], ra[l]) <= 1e-6, (key, kind, l)
        if psi.size:
            assert rel_l2(psi, rpsi) <= 1e-6, (key, kind)
        assert d.iteration == rd.iteration == steps - 1
        assert times[0] <= times[1] <= times[2] <= times[3]


def test_memory_budget_limits_concurrency():
    p, _, _ = fp32("mhd_hpml")
    res, peak = estimate_bytes(p)
    # one running (resident) and one in set-up (peak) fit; two running and
    # a third in set-up do not
    budget = res + peak + res // 2
    requests = [(0.0, k, fp32("mhd_hpml")[0], 0, 12) for k in range(5)]
    seen = []

    def build(key):
        _, bg, src = fp32("mhd_hpml")
        return bg, src

    def on_result(key, sim, state, times):
        seen.append(state)

    with Server(capacity=8, budget_bytes=budget, quantum=3) as srv:
        drive(srv, requests, build, on_result, deadline_s=200)
        st = srv.stats()
    assert seen == [abi.SPARC_REQ_DONE] * 5
    assert 1 <= st["max_concurrent"] <= 2
    assert st["point_updates"] == pytest.approx(5 * 12 * p.nx * p.ny * p.nz)


def test_request_above_budget_is_refused():
    p, _, _ = fp32("mhd_hpml")
    _, peak = estimate_bytes(p)
    with Server(capacity=2, budget_bytes=peak // 2) as srv:
        with pytest.raises(abi.SparcError) as e:
            srv.submit(p, 0, 10)
        assert e.value.code == abi.SPARC_ERR_NOMEM
