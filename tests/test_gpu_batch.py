"""The batched engine (sparc_batch_*) against the same simulations run alone.

A member's result must not depend on the company it keeps: every member of
a batch ends where the same SPARC_FP32 simulation run alone (sparc_run)
ends.  The batched kernels evaluate the same per-point arithmetic as the
single-simulation kernels, on other tile shapes (32x16 quiet tiles, the
cp.async MHD body), so the tolerance is FP32-level (1e-6 relative L2 per
field); the diagnostics' reduction order differs too.
"""
import numpy as np
import pytest

from sparc2_b200 import Simulation, abi
from sparc2_b200.batch import Batch
from tests import cases
from tests.cases import rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-6

MEMBERS = {
    "quiet_periodic": cases.quiet_periodic,
    "quiet_hpml": cases.quiet_hpml,
    "thermal_hpml": cases.thermal_hpml,
    "mhd_hpml": cases.mhd_hpml,
    "mhd_hpml_nx42": lambda: cases.mhd_hpml(nx=42, ny=40),
    "mhd_periodic": cases.mhd_periodic,
    "mhd_hpml_96": cases.CASES["mhd_hpml_96"],   # interior tiles: the batch's first part
    # PULSE = 0 members: their forcing planes are rebuilt each batched step
    "quiet_random": cases.quiet_random,
    "mhd_random": lambda: cases.mhd_random(nx=40, ny=40),
}


def fp32(name):
    p, bg, src = MEMBERS[name]()
    p.precision = abi.SPARC_FP32
    return p, bg, src


def alone(name, first, count):
    s = Simulation(*fp32(name))
    s.run(first, count)
    a, psi = s.get_state()
    d, r = s.diagnostics()
    s.close()
    return a, psi, d, r


def check(name, sim, ref):
    a, psi = sim.get_state()
    ra, rpsi, rd, rr = ref
    for l in range(sim.V):
        e = rel_l2(a[l], ra[l])
        assert e <= TOL, (name, l, e)
    if sim.n_psi:
        assert rel_l2(psi, rpsi) <= TOL, name
    d, r = sim.diagnostics()
    assert r == rr, name
    assert d.iteration == rd.iteration, name
    assert d.ke_norm == pytest.approx(rd.ke_norm, rel=1e-6), name


def test_batch_members_match_their_single_runs():
    counts = {n: 60 - 7 * i for i, n in enumerate(sorted(MEMBERS))}
    refs = {n: alone(n, 0, c) for n, c in counts.items()}
    with Batch(len(MEMBERS)) as b:
        sims = {}
        for n, c in counts.items():
            sims[n] = Simulation(*fp32(n))
            b.add(sims[n], 0, c)
        b.run(max(counts.values()) + 3)   # finished members stand still
        rem = b.remaining()
        assert sorted(rem[rem >= 0].tolist()) == [0] * len(counts)
        for slot in list(b.members):
            b.remove(slot)
    for n, s in sims.items():
        check(n, s, refs[n])


def test_staggered_admission_continuous_batching():
    """Members join and leave while others run; each result equals its run
    alone (the serving loop's invariance)."""
    plan = [("mhd_hpml", 0, 50, 0), ("quiet_periodic", 0, 40, 12),
            ("mhd_periodic", 0, 30, 20), ("thermal_hpml", 5, 25, 31)]
    refs = {n: alone(n, f, c) for n, f, c, _ in plan}
    sims = {}
    with Batch(3) as b:
        step = 0
        pending = sorted(plan, key=lambda t: t[3])
        live = {}
        while pending or live:
            while pending and pending[0][3] <= step and len(live) < 3:
                n, f, c, _ = pending.pop(0)
                sims[n] = Simulation(*fp32(n))
                live[b.add(sims[n], f, c)] = n
            b.run(1)
            step += 1
            rem = b.remaining()
            for slot in [q for q in live if rem[q] == 0]:
                b.remove(slot)
                live.pop(slot)
            assert step < 400
    for n, s in sims.items():
        check(n, s, refs[n])


def test_tile_extent_does_not_change_results():
    res = []
    for zm, zq in ((16, 16), (48, 150)):
        with Batch(2) as b:
            s1, s2 = Simulation(*fp32("mhd_hpml")), Simulation(*fp32("quiet_hpml"))
            b.set_tiles(zm, zq)
            b.add(s1, 0, 20)
            b.add(s2, 0, 20)
            b.run(20)
            for q in list(b.members):
                b.remove(q)
        res.append((s1.get_state()[0], s2.get_state()[0]))
    assert np.array_equal(res[0][0], res[1][0])
    assert np.array_equal(res[0][1], res[1][1])


def test_tuner_and_membership_rules():
    s = Simulation(*fp32("mhd_hpml"))
    q = Simulation(*fp32("quiet_periodic"))
    with Batch(2) as b:
        b.add(s, 0, 100)
        b.add(q, 0, 100)
        zm, zq = b.tune(steps_per_trial=1)
        assert zm >= 11 and zq >= 11
        assert b.tiles() == (zm, zq)
        with pytest.raises(abi.SparcError) as e:
            s.step(0)
        assert e.value.code == abi.SPARC_ERR_ORDER
        d, _ = s.diagnostics()          # allowed in a batch
        assert d.iteration >= 0
        p64, bg, src = cases.quiet_periodic()
        with pytest.raises(abi.SparcError):
            b.add(Simulation(p64, bg, src), 0, 10)   # FP64 handle
    s.step(200)                                      # usable alone again
