"""The largest single-field workload: 1536^2 x 512 (nx = 511, nz = 512,
ny = 512; 268.7 M spectral modes a component), Re 10000, dt 0.0005,
exact_shift, S2(t) = 0.5 sin(2 pi t / 10), the hard large-scale damping
mask (semi-axes 2, 2).  Far beyond what the oracle finishes, so the mixed
precision form is checked against the FP64 form on the same seeded field
(k0 = 24, energy 0.1) after 30 substeps: relative L2 of the velocity and
the energy and dissipation of outstats.  The two contexts (114 GB and 72 GB
of HBM) are created one after the other."""
import math

import numpy as np
import pytest

from homogenenousshearturbulence_b200 import hst
from tests.gpu_util import rel_l2

pytestmark = pytest.mark.gpu

DECK = dict(nx=511, ny=512, nz=512, alfa0=1.0, beta0=1.0, ly=2.0 * math.pi, re=10000.0, S=1.0, deltat=0.0005,
            cflmax=0.0, exact_shift=True, s2_amplitude=0.5, s2_period=10.0, damp_kpar=2.0, damp_kperp=2.0,
            damp_hard=True)
STEPS = 10  # time steps: 30 substeps


def run(prec, V0=None):
    s = hst.Solver(dict(DECK, precision=prec))
    try:
        if V0 is None:
            V0 = hst.random_field(DECK["nx"], DECK["ny"], DECK["nz"], DECK["alfa0"], DECK["beta0"], DECK["ly"], s.y,
                                  seed=5, k0=24.0, energy=0.1)
        s.set_velocity(V0)
        e0 = s.outstats()["energy"]
        for _ in range(STEPS):
            s.timestep()
        st = s.outstats()
        return V0, s.velocity(), st, e0, s.cfl
    finally:
        s.close()


def test_1536_mixed_precision_against_fp64():
    import psutil
    import torch
    free, _ = torch.cuda.mem_get_info(0)
    need = hst.device_bytes(**DECK)
    if free < 1.05 * need:
        pytest.skip(f"needs {need / 1e9:.0f} GB free on the device, {free / 1e9:.0f} GB free")
    if psutil.virtual_memory().available < 48e9:
        pytest.skip("needs about 48 GB of free host memory for the three 13 GB fields")
    V0, Vd, sd, e0, cfl_d = run("fp64")
    assert abs(e0 - 0.1) < 1e-6 * 0.1
    _, Vm, sm, _, cfl_m = run("mixed", V0)
    del V0
    assert np.isfinite(Vd).all() and np.isfinite(Vm).all()
    err = rel_l2(Vm, Vd)
    assert err <= 1e-5, err
    for k in ("energy", "diss"):
        assert abs(sm[k] - sd[k]) <= 1e-6 * abs(sd[k]), (k, sm[k], sd[k])
    assert abs(cfl_m - cfl_d) <= 1e-5 * cfl_d
