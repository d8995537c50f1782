"""An ensemble of independent realisations in one context
(hst_gpu_create_batch): every kernel of the substep covers all members in one
launch; each member must evolve exactly as it does alone in its own
context."""
import numpy as np
import pytest

from homogenenousshearturbulence_b200 import hst
from tests.gpu_util import c1_deck, rel_l2, seeded_field

pytestmark = pytest.mark.gpu

CASES = {
    "default": dict(),
    "exact_s2_edges": dict(exact_shift=True, s2_amplitude=0.5, s2_period=0.7),  # nzd = 3 nz: ghost-row transforms
    "mixed": dict(precision="mixed", exact_shift=True),
    "tall_persistent": dict(nx=15, nz=16, ny=512, exact_shift=True),  # 16-row slabs: the persistent solve stage
    "hard_damping": dict(damp_kpar=3.0, damp_kperp=2.0, damp_hard=True, s2_amplitude=0.4, s2_period=0.5),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_ensemble_members_match_single_contexts(case):
    """Three members with their own seeds, 5 time steps in one ensemble
    context against three single contexts: every member identical to 1e-15
    (the same kernels on the same data), the CFL number the largest of the
    members'."""
    deck = c1_deck(**CASES[case])
    fields = [seeded_field(deck, seed=s, k0=4.0, energy=0.1) for s in (1, 2, 3)]
    ens = hst.Solver(deck, members=3)
    assert hst.lib().hst_gpu_members(ens._h) == 3
    ens.time = 0.0
    for m, V in enumerate(fields):
        ens.select(m)
        ens.set_velocity(V)
    singles = []
    for V in fields:
        s = hst.Solver(deck)
        s.time = 0.0
        s.set_velocity(V)
        singles.append(s)
    for _ in range(5):
        ens.timestep(deck["deltat"])
        for s in singles:
            s.timestep(deck["deltat"])
    assert abs(ens.cfl - max(s.cfl for s in singles)) <= 1e-15 * ens.cfl
    for m, s in enumerate(singles):
        ens.select(m)
        err = rel_l2(ens.velocity(), s.velocity())
        assert err <= 1e-15, (case, m, err)
        s.close()
    ens.close()


def test_ensemble_refuses_bad_members():
    deck = c1_deck()
    ens = hst.Solver(deck, members=2)
    with pytest.raises(hst.HstError) as e:
        ens.select(2)
    assert e.value.code == hst.EARG
    with pytest.raises(hst.HstError):
        ens.autotune(deck["deltat"], 1)
    ens.close()
