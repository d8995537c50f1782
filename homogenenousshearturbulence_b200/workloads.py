"""The benchmark workloads: decks and seeded initial spectra.

Each single-field workload is a deck (the hst.in keys the Solver takes) and
the peak wavenumber k0 of its seeded divergence-free initial field (energy
spectrum E(k) ~ k^4 exp(-2 (k/k0)^2), energy 0.1, hst.random_field).  The
deck nx is the number of retained x modes minus one, so that the reference's
own padding (src/hst_input.f90:97-98) gives the stated dealiased grids.
The reference publishes no result for these decks: they are synthetic
inputs of the sizes the benchmark is quoted on.
"""
from __future__ import annotations

import math

PI = math.pi

WORKLOADS = {
    # 96^2 x 64, Re 1000, dt 0.005
    "c1": dict(deck=dict(nx=31, ny=64, nz=32, alfa0=1.0, beta0=1.0, ly=2 * PI, re=1000.0, S=1.0, deltat=0.005),
               k0=4.0, label="96x96 dealiased x 64 (nx=31, nz=32, ny=64), Re 1000, dt 0.005"),
    # 384^2 x 256, Re 2000, dt 0.002
    "c2": dict(deck=dict(nx=127, ny=256, nz=128, alfa0=1.0, beta0=1.0, ly=2 * PI, re=2000.0, S=1.0, deltat=0.002),
               k0=8.0, label="384x384 dealiased x 256 (nx=127, nz=128, ny=256), Re 2000, dt 0.002"),
    # 768^2 x 512 ("512^3"), Re 5000, dt 0.001, exact_shift
    "c3": dict(deck=dict(nx=255, ny=512, nz=256, alfa0=1.0, beta0=1.0, ly=2 * PI, re=5000.0, S=1.0, deltat=0.001,
                         exact_shift=True),
               k0=16.0, label="768x768 dealiased x 512 (nx=255, nz=256, ny=512), Re 5000, dt 0.001, exact_shift"),
    # 1536^2 x 512, Re 10000, dt 0.0005, exact_shift, S2(t) = 0.5 sin(2 pi t / 10), the hard large-scale damping
    # mask with semi-axes 2 following the shear angle
    "c5": dict(deck=dict(nx=511, ny=512, nz=512, alfa0=1.0, beta0=1.0, ly=2 * PI, re=10000.0, S=1.0, deltat=0.0005,
                         exact_shift=True, s2_amplitude=0.5, s2_period=10.0, damp_kpar=2.0, damp_kperp=2.0,
                         damp_hard=True),
               k0=24.0,
               label="1536x1536 dealiased x 512 (nx=511, nz=512, ny=512), Re 10000, dt 0.0005, exact_shift, "
                     "S2 = 0.5 sin(2 pi t/10), hard damping inside |k| < 2"),
}

# The ensemble of independent realisations with uneven sizes: 24 members of
# 192^2 x 128 (deck nx = 63, nz = 64, ny = 128) and 8 of 384^2 x 192 (nx = 95,
# nz = 96, ny = 192; the reference pads nxd, nzd to 192, 384), seeds 1..32,
# Re 1500, dt 0.004, k0 6, energy 0.1.
ENSEMBLE = [dict(nx=63, ny=128, nz=64)] * 24 + [dict(nx=95, ny=192, nz=96)] * 8
ENSEMBLE_COMMON = dict(alfa0=1.0, beta0=1.0, ly=2 * PI, re=1500.0, S=1.0, deltat=0.004)
ENSEMBLE_K0 = 6.0


def seeded_field(name: str, y, seed: int = 1):
    """The workload's initial field on the grid y(-2:ny+1)."""
    from homogenenousshearturbulence_b200 import hst
    w = WORKLOADS[name]
    d = w["deck"]
    return hst.random_field(d["nx"], d["ny"], d["nz"], d["alfa0"], d["beta0"], d["ly"], y, seed=seed, k0=w["k0"],
                            energy=0.1)
