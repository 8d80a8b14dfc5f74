"""Regenerates the golden fixtures of the oracle (tests/golden/*.npz).

Run from the repository root:  python tests/golden/make_golden.py [NAME...]
(all fixtures without names).
The fixtures freeze the oracle's output on tiny seeded cases so that any
change of the restatement is deliberate.  Each fixture keeps, per state
field, the L2 norm, sum, max |.| and the x-y slice at the middle layer, plus
the same for the CPML auxiliary state and the diagnostics.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from tests import cases  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))

FIXTURES = {
    # name: (case, kwargs, random-state seed or None, first iteration, count)
    "quiet_rest_12": ("quiet_periodic", dict(nx=24, ny=24, nz=32, npml=6), None, 0, 12),
    "mhd_rest_12": ("mhd_hpml", dict(nx=24, ny=24, nz=32, npml=6, npulses=8), None, 0, 12),
    "quiet_random_it30": ("quiet_periodic", dict(nx=24, ny=24, nz=32, npml=6), 21, 30, 1),
    "mhd_random_it30": ("mhd_hpml", dict(nx=24, ny=24, nz=32, npml=6, npulses=8), 22, 30, 1),
    # PULSE = 0 random-series source from rest (the series' first samples
    # are dropped at early times, as LAGRANGE_INTERP does)
    "quiet_rndsrc_40": ("quiet_random", dict(nx=24, ny=24, nz=32), None, 0, 40),
}


def summarize(o):
    a, psi = o.get_state()
    d, r = o.diagnostics()
    k = a.shape[1] // 2
    return dict(
        l2=np.sqrt(np.sum(a ** 2, axis=(1, 2, 3))),
        sum=np.sum(a, axis=(1, 2, 3)),
        maxabs=np.max(np.abs(a), axis=(1, 2, 3)),
        slice=a[:, k].copy(),
        psi_l2=np.array([np.sqrt(np.sum(psi ** 2))]),
        psi_head=psi[:256].copy(),
        diag=np.array([d.ke_norm, d.min_rho, d.min_p, d.iteration,
                       d.fail_iteration, r], dtype=np.float64),
    )


def run(name):
    case, kw, seed, first, count = FIXTURES[name]
    p, bg, src = cases.CASES[case](**kw)
    o = oracle.Oracle(p, bg, src)
    if seed is not None:
        a0, psi0 = cases.random_state(o, seed)
        o.set_state(a0, psi0)
    o.run(first, count)
    return summarize(o)


def main(names=None):
    oracle.build()
    for name in names or FIXTURES:
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **run(name))
        print("wrote", name)


if __name__ == "__main__":
    main(sys.argv[1:])
