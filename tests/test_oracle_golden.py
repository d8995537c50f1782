"""The oracle against the reference's own golden fields.

tests/regression.sh of the reference runs the decks small, small_s2x and
small_stokes for 50 steps and compares the final Dati.cart.out with
tests/reference/<deck>.fld at 1e-10 max-abs relative over the interior
rows (tests/compare_fields.py:51-57).  The oracle must pass the same gate;
this pins it before it is trusted as the checker of the CUDA path.
"""
import hashlib

import numpy as np
import pytest

import oracle


def test_fixture_checksums(golden):
    for line in (golden / "SHA256SUMS").read_text().splitlines():
        digest, name = line.split()
        assert hashlib.sha256((golden / name).read_bytes()).hexdigest() == digest, name


@pytest.mark.parametrize("deck", ["small", "small_s2x", "small_stokes"])
def test_regression_field(golden, deck, tmp_path):
    p = oracle.read_deck(golden / f"{deck}.in")
    p.restart_from_file = 0          # the reference run starts from no restart file: generated field
    s = oracle.Sim(p)
    s.start()
    n = s.run(10**9)
    assert n == 50
    out = tmp_path / "out.fld"
    assert s.restart_write(out) == 0
    t_ref, ref = oracle.read_cpl(golden / f"{deck}.fld")
    t_new, new = oracle.read_cpl(out)
    assert t_new == t_ref
    rel = oracle.cpl_compare(new, ref)
    assert rel <= 1e-10, rel


def test_uniform_from_key_properties():
    # the keyed deviate: a pure function of its keys, in [0, 1), (src/hst_initial.f90:139-159)
    u = [oracle.uniform_from_key(1, c, m, iz, ix) for c in range(1, 4) for m in (-3, 0, 5) for iz in (-2, 7)
         for ix in (0, 3)]
    assert all(0.0 <= x < 1.0 for x in u)
    assert len(set(u)) == len(u)
    assert oracle.uniform_from_key(1, 2, -3, 7, 3) == oracle.uniform_from_key(1, 2, -3, 7, 3)


def taylor_green_pressure_case(golden, Sim, params_of):
    """The reference's tests/test_pressure.f90 set-up: u = cos(kx) sin(ky),
    v = -sin(kx) cos(ky), w = 0 at k = 3 alfa0 = 2 pi 2/ly (S = 0).  Returns
    (ix = 2mx mode of p, (0,0) mode of p, every other mode, y)."""
    from homogenenousshearturbulence_b200 import hst
    deck = hst.read_deck(golden / "pressure.in")
    deck["S"] = 0.0
    o = Sim(params_of(deck))
    y = o.y()
    mx = 3
    ky = mx * deck["alfa0"]
    shape = o.field(0).shape
    U = np.zeros(shape, np.complex128)
    Vv = np.zeros(shape, np.complex128)
    U[mx, deck["nz"], :] = 0.5 * np.sin(ky * y)
    Vv[mx, deck["nz"], :] = 0.5j * np.cos(ky * y)
    return deck, o, U, Vv, ky, y


def test_oracle_pressure_taylor_green(golden):
    """compute_pressure of the oracle passes the reference's Taylor-Green
    pressure test (tests/test_pressure.f90): the two nonzero modes
    p(2mx, 0) = -1/8 and p(0,0)(y) = -cos(2ky)/4 within 1e-4, every other
    mode below 1e-10."""
    from tests.gpu_util import deck_to_oracle
    deck, o, U, Vv, ky, y = taylor_green_pressure_case(golden, oracle.Sim, deck_to_oracle)
    o.time = 0.0
    o.field(oracle.V1)[...] = U
    o.field(oracle.V2)[...] = Vv
    o.field(oracle.V3)[...] = 0
    for c in range(3):
        o.fill_ghosts(c)
    o.compute_pressure(oracle.RHS2)
    p = o.field(oracle.RHS2)[..., 2:-2]
    nz, mx = deck["nz"], 3
    err = max(np.abs(p[2 * mx, nz] + 0.125).max(), np.abs(p[0, nz] + 0.25 * np.cos(2 * ky * y[2:-2])).max())
    other = p.copy()
    other[2 * mx, nz] = 0
    other[0, nz] = 0
    assert err <= 1e-4, err
    assert np.abs(other).max() <= 1e-10
