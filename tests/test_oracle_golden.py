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
