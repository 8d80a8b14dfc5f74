"""Generates the oracle fixture of the flux-tube configuration at full depth.

Run from the repository root:  python tests/golden/make_fluxtube_1000.py
(about an hour on 8 host cores; writes tests/golden/fluxtube_96x96x300.npz).

Physics of the 256x256x300 flux tube (z from -25 to +1 Mm over 300 layers,
CPML 10 points on all six faces, Alfven speed capped at 40 km/s, seeded PSR
pulse table, dt = 0.5 s, z filter every 10 iterations and xy filter every
30, rank layout 2x2x4) on 96x96 columns at the same horizontal spacing
(37.5 Mm), run for 1000 driver iterations from rest (driver.f90:123-202).
96 columns give interior stage tiles as well as edge and CPML tiles, and
300 layers give several z chunks with the top one-sided rows under a chunk
seam.

The full state (2.2e7 values) is too large to commit, so the fixture keeps,
at iterations 100, 500 and 1000 (after the iteration's filter):
  * per field: the exact L2 norm, sum and max |.| over the whole grid;
  * a sample of every field at the flattened indices 0, S, 2S, ... (S = 307,
    a prime, so the sample crosses every layer, row and column class);
    the relative L2 error over the sample estimates the full-field error;
  * the CPML auxiliary state: its exact L2 norm and the same strided sample;
and the diagnostics (KE norm, min rho, min p) of every iteration.
"""
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from sparc2_b200 import workloads as W  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
NAME = "fluxtube_96x96x300"
STRIDE = 307
CHECKPOINTS = (100, 500, 1000)
NXY, NZ = 96, 300


def config():
    """(params, background, source) of the fixture: the flux-tube preset on
    96x96 columns at its horizontal spacing (100 Mm / 256 points)."""
    return W.cfg1(nx=NXY, ny=NXY, nz=NZ, length_mm=NXY * 100.0 / 256.0)


def sample(a, psi):
    """The fixture's view of a state (V, nz, ny, nx) and CPML vector."""
    V = a.shape[0]
    flat = a.reshape(V, -1)
    return dict(
        l2=np.sqrt(np.sum(a * a, axis=(1, 2, 3))),
        sum=np.sum(a, axis=(1, 2, 3)),
        maxabs=np.max(np.abs(a), axis=(1, 2, 3)),
        samp=flat[:, ::STRIDE].copy(),
        psi_l2=np.array([np.sqrt(np.sum(psi * psi))]),
        psi_samp=psi[::STRIDE].copy(),
    )


def main():
    import oracle
    oracle.build()
    p, bg, src = config()
    o = oracle.Oracle(p, bg, src)
    out = {}
    diag = np.zeros((CHECKPOINTS[-1], 3))
    t0 = time.time()
    for nn in range(CHECKPOINTS[-1]):
        o.run(nn, 1)
        d, r = o.diagnostics()
        if r != 0:
            raise SystemExit(f"oracle reports failure at iteration {nn}")
        diag[nn] = (d.ke_norm, d.min_rho, d.min_p)
        if nn + 1 in CHECKPOINTS:
            a, psi = o.get_state()
            for k, v in sample(a, psi).items():
                out[f"it{nn + 1}_{k}"] = v
            print(f"iteration {nn + 1}: {time.time() - t0:.0f} s", flush=True)
    out["diag"] = diag
    out["stride"] = np.array([STRIDE])
    np.savez_compressed(os.path.join(HERE, NAME + ".npz"), **out)
    print("wrote", NAME)


if __name__ == "__main__":
    main()
