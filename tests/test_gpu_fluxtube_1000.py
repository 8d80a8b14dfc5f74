"""The flux-tube configuration at full depth against the oracle fixture
(tests/golden/fluxtube_96x96x300.npz, written by make_fluxtube_1000.py):
1000 driver iterations from rest (driver.f90:123-202) on 96x96x300 columns
with CPML on all six faces, the seeded PSR pulse table and both filters.

The fixture holds, at iterations 100, 500 and 1000, exact full-grid norms
and a strided sample (every 307th value) of each state field and of the
CPML auxiliary state, plus the oracle's diagnostics of every iteration.

Tolerances:
  * FP64 plain form: relative L2 per field over the sample, relative
    difference of the full-grid L2 norms, CPML state and every iteration's
    KE norm, all <= 1e-11 (the plain form's bar after 1000 steps).
  * FP32 precision form: relative L2 per field over the sample <= 1e-4 at
    each checkpoint; the relative L2 and max-norm errors are printed.
"""
import os

import numpy as np
import pytest

from sparc2_b200 import Simulation, abi
from tests.cases import rel_l2
from tests.golden import make_fluxtube_1000 as F

pytestmark = pytest.mark.gpu

FIXTURE = os.path.join(os.path.dirname(__file__), "golden", F.NAME + ".npz")
FP64_TOL = 1e-11
FP32_TOL = 1e-4
FIELDS = ["rho", "vx", "vy", "vz", "p", "bx", "by", "bz"]


@pytest.fixture(scope="module")
def ref():
    return dict(np.load(FIXTURE))


def run_against(ref, precision):
    """Runs the fixture's configuration for 1000 iterations; returns the
    per-iteration KE norms and, per checkpoint, the sample of the state."""
    p, bg, src = F.config()
    p.precision = precision
    sim = Simulation(p, bg, src)
    ke = np.zeros(F.CHECKPOINTS[-1])
    snaps = {}
    for nn in range(F.CHECKPOINTS[-1]):
        sim.run(nn, 1)
        d, r = sim.diagnostics()
        assert r == abi.SPARC_OK, (nn, r)
        ke[nn] = d.ke_norm
        if nn + 1 in F.CHECKPOINTS:
            a, psi = sim.get_state()
            snaps[nn + 1] = F.sample(a, psi)
    sim.close()
    return ke, snaps


def errors(ref, snap, it):
    """(relative L2, max-norm relative to max |ref|) per field over the
    sample at checkpoint it."""
    out = []
    for l in range(snap["samp"].shape[0]):
        g, o = snap["samp"][l], ref[f"it{it}_samp"][l]
        mx = np.max(np.abs(o))
        out.append((rel_l2(g, o), np.max(np.abs(g - o)) / mx if mx > 0 else np.max(np.abs(g))))
    return out


def test_fixture_shape(ref):
    assert ref["stride"][0] == F.STRIDE
    assert ref["diag"].shape == (F.CHECKPOINTS[-1], 3)
    for it in F.CHECKPOINTS:
        assert ref[f"it{it}_samp"].shape[0] == 8


def test_fp64_plain_1000_iterations(ref):
    ke, snaps = run_against(ref, abi.SPARC_FP64)
    kref = ref["diag"][:, 0]
    live = kref > 0
    assert np.all(live[1:])
    assert np.max(np.abs(ke[live] - kref[live]) / kref[live]) <= FP64_TOL
    for it in F.CHECKPOINTS:
        s = snaps[it]
        for l, (e2, emax) in enumerate(errors(ref, s, it)):
            assert e2 <= FP64_TOL, (it, FIELDS[l], e2, emax)
        rl2 = np.abs(s["l2"] - ref[f"it{it}_l2"]) / ref[f"it{it}_l2"]
        assert np.max(rl2) <= FP64_TOL, (it, rl2)
        assert rel_l2(s["psi_samp"], ref[f"it{it}_psi_samp"]) <= FP64_TOL
        assert abs(s["psi_l2"][0] - ref[f"it{it}_psi_l2"][0]) <= \
            FP64_TOL * ref[f"it{it}_psi_l2"][0]


def test_fp32_precision_form_against_the_oracle(ref):
    ke, snaps = run_against(ref, abi.SPARC_FP32)
    for it in F.CHECKPOINTS:
        errs = errors(ref, snaps[it], it)
        print(f"FP32 vs FP64 oracle, iteration {it}: " + ", ".join(
            f"{FIELDS[l]} {e2:.2e}/{em:.2e}" for l, (e2, em) in enumerate(errs)))
        for l, (e2, _) in enumerate(errs):
            assert e2 <= FP32_TOL, (it, FIELDS[l], e2)
    kref = ref["diag"][:, 0]
    assert np.max(np.abs(ke[1:] - kref[1:]) / kref[1:]) <= FP32_TOL
