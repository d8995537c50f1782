"""The solve stage's forms: the one-kernel solves (HST_SOLVE_HALVES=0, read
when a context is created) and the same solves as two one-line passes (the
default where the context has its global factor scratch) must give the same
bits, since they run the same operations in the same order; the halves
against the oracle as well."""
import os

import numpy as np
import pytest

from tests.gpu_util import c1_deck, make_pair, rel_l2, run_pair, seeded_field
from homogenenousshearturbulence_b200 import hst

pytestmark = pytest.mark.gpu

CASES = {
    # 512 rows: 16-row slabs, the persistent solve stage with its global factor scratch
    "exact": dict(nx=15, nz=16, ny=512, exact_shift=True),
    "default_s2": dict(nx=15, nz=16, ny=512, s2_amplitude=0.5, s2_period=0.7),
    "exact_mixed": dict(nx=31, nz=32, ny=512, exact_shift=True, precision="mixed"),  # 2 nxd = nzd = 96
    "hard_damping": dict(nx=15, nz=16, ny=512, damp_kpar=3.0, damp_kperp=2.0, damp_hard=True, exact_shift=True),
}


FORMS = {"one_pass": dict(HST_SOLVE_HALVES="0"), "halves": dict(HST_SOLVE_HALVES="1")}


def solver_with(deck, form, V0):
    env = FORMS[form]
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        s, o = make_pair(deck, V0)
    finally:
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v
    return s, o


@pytest.mark.parametrize("form", ["halves"])
@pytest.mark.parametrize("case", sorted(CASES))
def test_solve_forms_same_bits(case, form):
    """3 time steps of a 512-row deck with the solves in one pass and in two
    halves: identical velocity bits and CFL number; the halves within the
    precision's bound of the oracle."""
    deck = c1_deck(**CASES[case])
    V0 = seeded_field(deck, seed=6, k0=4.0, energy=0.1)
    s1, _ = solver_with(deck, "one_pass", V0)
    s2, o = solver_with(deck, form, V0)
    for _ in range(3):
        s1.timestep(deck["deltat"])
    V2, Vo = run_pair(s2, o, deck["deltat"], 3)
    V1 = s1.velocity()
    assert np.array_equal(V1, V2), np.abs(V1 - V2).max()
    assert s1.cfl == s2.cfl
    tol = 1e-5 if deck.get("precision") == "mixed" else 1e-12
    assert rel_l2(V2, Vo) <= tol
    s1.close()
    s2.close()
