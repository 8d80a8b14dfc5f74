"""DAMPING (all_modules.f90:1803-1888 damp_velocity, rates of
initialize.f90:1276-1340 INIT_DAMPING) in the oracle, pinned against numpy's
FFT: the RHS with damping minus the RHS without is -term on the three
velocities and nothing elsewhere, term(:,:,k) = c2r(r2c(v(:,:,k)) * rates)
with unnormalised transforms, the rates written out here from the
reference's expression."""
import numpy as np
import pytest

import oracle
from sparc2_b200 import abi
from tests import cases

RSUN = 69598946770.0
PI_REF = 3.14159265358979


def rates_of(p, dimc):
    nx, ny = p.nx, p.ny
    nh = nx // 2 + 1
    constx = 2.0 * PI_REF * RSUN / p.xlength
    consty = 2.0 * PI_REF * RSUN / p.ylength
    i = np.arange(nh, dtype=np.float64)
    j = np.arange(ny)
    ky = np.where(j <= ny // 2, j, ny - j).astype(np.float64)
    kay = (constx * constx * (i[None, :] * i[None, :])
           + consty * consty * (ky[:, None] * ky[:, None])) ** 0.5
    return RSUN / dimc / nx / ny * 1.0e-6 * (500.0 * (kay / 902.0) ** 2.2) * 20.0


@pytest.mark.parametrize("name,kw", [("quiet_periodic", {}), ("mhd_hpml", {"nx": 41})])
def test_damping_term_matches_numpy_fft(name, kw):
    p, bg, src = cases.CASES[name](**kw)
    off = oracle.Oracle(p, bg, src)
    p2, _, _ = cases.CASES[name](**kw)
    p2.damping = 1
    on = oracle.Oracle(p2, bg, src)
    a, psi = cases.random_state(off, seed=21)
    r0, _ = off.rhs(3, a, psi)
    r1, _ = on.rhs(3, a, psi)
    V = off.V
    shape = (V, p.nz, p.ny, p.nx)
    d = (r1 - r0).reshape(shape)
    dimc = off.scalars()["dimc"]
    rates = rates_of(p, dimc)
    for l in range(V):
        if l in (1, 2, 3):
            v = a.reshape(shape)[l]
            spec = np.fft.rfft2(v, axes=(1, 2)) * rates[None]
            term = np.fft.irfft2(spec, s=(p.ny, p.nx), axes=(1, 2)) * (p.nx * p.ny)
            scale = np.max(np.abs(term))
            assert scale > 0
            assert np.max(np.abs(d[l] + term)) <= 1e-10 * scale + 1e-13 * np.max(np.abs(r0)), l
        else:
            assert np.array_equal(d[l], np.zeros_like(d[l])), l


def test_damping_flag_is_validated():
    p, bg, src = cases.quiet_periodic()
    p.damping = 2
    with pytest.raises(abi.SparcError):
        oracle.Oracle(p, bg, src)
