"""Helpers shared by the GPU tests: building matching oracle and GPU runs."""
import math

import numpy as np

import oracle
from homogenenousshearturbulence_b200 import hst

PI = math.pi


def deck_to_oracle(deck: dict) -> "oracle.Params":
    return oracle.params_from_deck(deck)


def interior(a):
    return a[..., 2:-2]


def rel_l2(a, b):
    """relative L2 over the interior rows; absolute when b is zero there"""
    nb = np.linalg.norm(interior(b))
    d = np.linalg.norm(interior(a) - interior(b))
    return float(d / nb) if nb > 0 else float(d)


def rel_maxabs(a, b):
    """the reference's compare_fields metric: max |A-B| over the interior rows / max |B|"""
    return float(np.abs(interior(a) - interior(b)).max() / np.abs(b).max())


def make_pair(deck: dict, V0: np.ndarray, device=0):
    """A GPU solver and an oracle run starting from the same field V0
    (3, nx+1, 2nz+1, ny+4) with ghost rows filled at t = time."""
    s = hst.Solver(deck, device=device)
    s.time = float(deck.get("time", 0.0))
    s.set_velocity(V0)
    o = oracle.Sim(deck_to_oracle(deck))
    o.time = s.time
    for c in range(3):
        o.field(c)[...] = V0[c]
        o.fill_ghosts(c)
    return s, o


def run_pair(s, o, dt, nsteps):
    o.deltat = dt
    for _ in range(nsteps):
        s.timestep(dt)
        o.timestep()
    Vg = s.velocity()
    Vo = np.stack([o.field(c).copy() for c in range(3)])
    return Vg, Vo


def c1_deck(**over):
    """The 96^2 x 64 workload (deck nx = 31, nz = 32, ny = 64): ly = 2 pi, alfa0 = beta0 = 1, Re = 1000, dt = 0.005."""
    d = dict(nx=31, ny=64, nz=32, alfa0=1.0, beta0=1.0, ly=2.0 * PI, re=1000.0, S=1.0, deltat=0.005, cflmax=0.0)
    d.update(over)
    return d


def seeded_field(deck, seed=1, k0=4.0, energy=0.1):
    s_y = oracle.Sim(deck_to_oracle(deck)).y()
    return hst.random_field(deck["nx"], deck["ny"], deck["nz"], deck["alfa0"], deck["beta0"], deck["ly"], s_y,
                            seed=seed, k0=k0, energy=energy)
