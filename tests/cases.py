"""Small seeded cases shared by the tests (sizes the oracle finishes in
seconds).  Each returns (params, background, source)."""
import numpy as np

from sparc2_b200 import abi
from sparc2_b200 import workloads as W

MM = W.MM


def quiet_periodic(nx=32, ny=32, nz=48, npml=10):
    """cfg0 physics on a small grid: periodic, z-CPML, v_z pulse."""
    p = W.base_params(nx, ny, nz, magnetic=0, periodic=True, hpml=False,
                      xlength=25.0 * MM, ylength=25.0 * MM, timestep=1.0,
                      t_z=10.0, t_xy=30.0, npml=npml, blocks=(2, 2, 2))
    bg = W.quiet_background(nx, ny, nz, -10.0, 1.0)
    src = W.pulse_source(px=0.5 * p.xlength, py=0.5 * p.ylength,
                         pz=-0.5 * MM, sr=1.5 * MM, sz=0.5 * MM, t1=20.0,
                         st=10.0)
    return p, bg, src


def _tube(nx, ny, nz, L, periodic):
    return W.fluxtube_background(nx, ny, nz, L, L, -6.0, 1.0, B0=3000.0,
                                 R0_mm=2.0, periodic=periodic)


def mhd_hpml(nx=40, ny=40, nz=48, npml=8, npulses=20, seed=11):
    """cfg1 physics on a small grid: flux tube, CPML on six faces, PSR."""
    L = 16.0 * MM
    p = W.base_params(nx, ny, nz, magnetic=2, periodic=False, hpml=True,
                      xlength=L, ylength=L, timestep=0.5, t_z=5.0, t_xy=15.0,
                      npml=npml, blocks=(2, 2, 2), maxva=4.0e6)
    bg = _tube(nx, ny, nz, L, False)
    tab = W.psr_table(p, npulses, seed)
    return p, bg, W.psr_source(tab)


def mhd_periodic(nx=32, ny=32, nz=48, npml=8):
    L = 16.0 * MM
    p = W.base_params(nx, ny, nz, magnetic=2, periodic=True, hpml=False,
                      xlength=L, ylength=L, timestep=0.5, t_z=5.0, t_xy=15.0,
                      npml=npml, blocks=(2, 2, 2), maxva=4.0e6)
    bg = _tube(nx, ny, nz, L, True)
    src = W.pulse_source(px=0.3 * L, py=0.6 * L, pz=-1.0 * MM, sr=1.0 * MM,
                         sz=0.4 * MM, t1=10.0, st=5.0, direction=1)
    return p, bg, src


def quiet_hpml(nx=40, ny=36, nz=48, npml=8):
    """Quiet background, non-periodic with side CPML (3-D coefficient
    path of the quiet kernel, x/y faces with two auxiliary fields)."""
    L = 16.0 * MM
    p = W.base_params(nx, ny, nz, magnetic=0, periodic=False, hpml=True,
                      xlength=L, ylength=L, timestep=1.0, t_z=10.0, t_xy=30.0,
                      npml=npml, blocks=(2, 2, 2))
    bg = W.quiet_background(nx, ny, nz, -8.0, 1.0)
    src = W.pulse_source(px=0.4 * L, py=0.5 * L, pz=-1.0 * MM, sr=1.0 * MM,
                         sz=0.5 * MM, t1=10.0, st=5.0, direction=2)
    return p, bg, src


def thermal_hpml(nx=40, ny=40, nz=48, npml=8, npulses=12, seed=5):
    """MAGNETIC = 1: quiet equations on the 3-D flux-tube thermodynamics."""
    L = 16.0 * MM
    p = W.base_params(nx, ny, nz, magnetic=1, periodic=False, hpml=True,
                      xlength=L, ylength=L, timestep=0.5, t_z=5.0, t_xy=15.0,
                      npml=npml, blocks=(2, 2, 2))
    bg = _tube(nx, ny, nz, L, False)
    bg = dict(bg, bx0=None, by0=None, bz0=None)
    tab = W.psr_table(p, npulses, seed)
    return p, bg, W.psr_source(tab)


def _random(p, seed, cad):
    """PULSE = 0 source: a seeded forcing series sampled every `cad` s."""
    series = W.random_series(p, 400, cad, seed)
    return W.random_source(series, cadforcing=cad, ampl=3.0e3, depth=-0.5 * MM,
                           sigma=0.3 * MM)


def quiet_random(nx=40, ny=36, nz=48):
    """Quiet background with side CPML, driven by the random source."""
    p, bg, _ = quiet_hpml(nx, ny, nz)
    return p, bg, _random(p, 21, 8.0)


def mhd_random(nx=96, ny=96, nz=48):
    """Flux tube with CPML on six faces (interior tiles too), driven by the
    random source."""
    p, bg, _ = mhd_hpml(nx, ny, nz)
    return p, bg, _random(p, 23, 4.0)


CASES = {
    "quiet_periodic": quiet_periodic,
    "quiet_hpml": quiet_hpml,
    "thermal_hpml": thermal_hpml,
    "mhd_hpml": mhd_hpml,
    "mhd_periodic": mhd_periodic,
    # 96x96 columns: 32x8 MHD tiles away from every edge and CPML slab
    # exist (x tile 32..63, y tiles 8..87), so the interior stage kernel
    # (and in FP64 its TMA halo planes) runs, not only the edge kernel
    "mhd_hpml_96": lambda: mhd_hpml(nx=96, ny=96, nz=48),
    "mhd_periodic_96": lambda: mhd_periodic(nx=96, ny=96, nz=48),
    "quiet_random": quiet_random,
    "mhd_random": mhd_random,
}


def random_state(sim_like, seed, amp=1.0e-3):
    rng = np.random.Generator(np.random.Philox(key=seed))
    a = amp * rng.standard_normal((sim_like.V,) + sim_like.shape)
    psi = amp * rng.standard_normal(sim_like.n_psi)
    return a, psi


def rel_l2(x, ref):
    """Relative L2 error per field (absolute where the reference is 0)."""
    x = np.asarray(x, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    num = np.sqrt(np.sum((x - ref) ** 2))
    den = np.sqrt(np.sum(ref ** 2))
    return num / den if den > 0 else num
