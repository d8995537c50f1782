"""The seeded initial field (hst.random_field, src/hst_initial.f90:27-67,
113-159) draws only the modes inside the box where its envelope is above the
1e-8 cut; here it is checked against the same field drawn over every mode
(|m| <= ny/3, all ix, iz), on the CPU."""
import math

import numpy as np
import pytest

from homogenenousshearturbulence_b200 import hst

PI = math.pi


def full_range_field(nx, ny, nz, alfa0, beta0, ly, y, seed, k0, envelope):
    mmax = ny // 3
    ix = np.arange(nx + 1)[:, None, None]
    iz = np.arange(-nz, nz + 1)[None, :, None]
    m = np.arange(-mmax, mmax + 1)[None, None, :]
    kx, kz, ky = alfa0 * ix, beta0 * iz, 2.0 * PI * m / ly
    k = np.sqrt(kx * kx + ky * ky + kz * kz)
    q = k / k0
    with np.errstate(divide="ignore", invalid="ignore"):
        env = np.exp(-q * q) if envelope == "gauss" else q * q * np.exp(1.0 - q * q)
    env = np.where((k == 0.0) | (env < 1e-8), 0.0, env)
    env = np.where((ix == 0) & (iz == 0), 0.0, env)
    mirror = (ix == 0) & ((iz < 0) | ((iz == 0) & (m < 0)))
    jz, jm = np.where(mirror, -iz, iz), np.where(mirror, -m, m)
    a = []
    for c in range(1, 4):
        r = hst.uniform_from_key(seed, c, jm, jz, ix)
        ph = 2.0 * PI * hst.uniform_from_key(seed, c + 3, jm, jz, ix)
        ac = r * np.exp(1j * ph)
        a.append(np.where(mirror, np.conj(ac), ac) * env)
    u = [1j * (ky * a[2] - kz * a[1]), 1j * (kz * a[0] - kx * a[2]), 1j * (kx * a[1] - ky * a[0])]
    E = np.exp(1j * ky[0, 0, :, None] * y[None, :])
    V = np.stack([np.einsum("xzm,my->xzy", uc, E) for uc in u])
    e = hst.box_energy(V, ly, y)
    return V * math.sqrt(0.1 / e)


@pytest.mark.parametrize("case", [
    dict(nx=31, ny=64, nz=32, alfa0=1.0, beta0=1.0, ly=2 * PI, k0=4.0, envelope="gauss"),
    dict(nx=63, ny=96, nz=48, alfa0=1.0, beta0=1.0, ly=2 * PI, k0=3.0, envelope="gauss"),
    dict(nx=47, ny=64, nz=40, alfa0=2 * PI / 3, beta0=2 * PI, ly=2.0, k0=4.0, envelope="hst"),
    dict(nx=15, ny=32, nz=16, alfa0=1.0, beta0=1.0, ly=2 * PI, k0=20.0, envelope="gauss"),  # box = every mode
])
def test_box_restricted_field_matches_full_range(case):
    c = dict(case)
    k0, envelope = c.pop("k0"), c.pop("envelope")
    ny, ly = c["ny"], c["ly"]
    y = (np.arange(-2, ny + 2) * (ly / ny))
    got = hst.random_field(c["nx"], ny, c["nz"], c["alfa0"], c["beta0"], ly, y, seed=7, k0=k0, energy=0.1,
                           envelope=envelope)
    want = full_range_field(c["nx"], ny, c["nz"], c["alfa0"], c["beta0"], ly, y, 7, k0, envelope)
    assert got.shape == want.shape
    assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()
    assert abs(hst.box_energy(got, ly, y) - 0.1) < 1e-12
