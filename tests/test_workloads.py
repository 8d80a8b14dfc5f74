"""Seeded synthetic inputs: reproducibility and physical sanity (CPU)."""
import numpy as np

from sparc2_b200 import workloads as W


def test_polytrope_is_hydrostatic():
    z = np.linspace(-20, 1, 2001)
    rho, pre, cs, g, _ = W.polytrope_1d(z)
    dpdz = np.gradient(pre, z * W.MM)
    mid = slice(5, -5)
    assert np.allclose(dpdz[mid], -rho[mid] * g[mid], rtol=5e-3)
    r0, _, _, _, _ = W.polytrope_1d(np.array([0.0]))
    assert r0[0] == 2e-7
    assert np.allclose(cs ** 2, 5.0 / 3.0 * pre / rho)


def test_fluxtube_is_divergence_free_and_positive():
    nx = ny = 64
    nz = 80
    L = 40.0 * W.MM
    bg = W.fluxtube_background(nx, ny, nz, L, L, -10.0, 1.0)
    bx, by, bz = bg["bx0"], bg["by0"], bg["bz0"]
    dx = L / (nx - 1)
    dz = (bg["zaxis"][1] - bg["zaxis"][0]) * W.MM
    div = (np.gradient(bx, dx, axis=2) + np.gradient(by, dx, axis=1) +
           np.gradient(bz, dz, axis=0))
    scale = np.abs(bz).max() / dz
    assert np.max(np.abs(div[2:-2, 2:-2, 2:-2])) < 0.05 * scale
    assert np.all(bg["pre0"] > 0) and np.all(bg["rho0"] > 0)
    assert abs(bz[:, ny // 2, nx // 2].max() - bz.max()) == 0.0


def test_psr_table_is_seeded_and_in_range():
    p, _, _ = W.cfg1(nx=64, ny=64, nz=60, npulses=10)
    t1 = W.psr_table(p, 50, seed=123)
    t2 = W.psr_table(p, 50, seed=123)
    t3 = W.psr_table(p, 50, seed=124)
    assert np.array_equal(t1, t2)
    assert not np.array_equal(t1, t3)
    # all_modules.f90:566-584 ranges
    assert np.all(t1["px"] >= p.npml_xb / p.nx)
    assert np.all(t1["px"] <= 1 - p.npml_xt / p.nx)
    depth_mm = (1.0 - t1["pz"]) * W.RSUN / W.MM
    assert np.all((depth_mm >= 0.1 - 1e-9) & (depth_mm <= 2.0 + 1e-9))
    assert np.all(t1["t0"] > 0) and np.all(t1["sr"] > 0)
