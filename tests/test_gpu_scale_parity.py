"""Parity with the oracle at the sizes the benchmark times.

The GPU substep and the oracle (the CPU FP64 restatement of the reference's
path) start from the same seeded field of the benchmark workload and run 30
substeps; the velocity must agree to 1e-12 relative L2 over the interior rows
in FP64 and to 1e-5 in mixed precision (the two targets the acceptance
states).  One oracle run serves both precisions.  This covers the transform
plans those sizes select: the 384-point z plans of the 384^2 x 256 workload
and the 768-point x and z plans and the 512-row line solves of the 768^2 x 512
exact_shift workload (and, on narrow decks, each 768-point direction with an
oscillating S2 as well).
"""
import math

import numpy as np
import pytest

import oracle
from homogenenousshearturbulence_b200 import hst
from homogenenousshearturbulence_b200.workloads import WORKLOADS, seeded_field
from tests.gpu_util import c1_deck, make_pair, rel_l2, run_pair

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
MIXED_TOL = 1e-5


def host_bytes_available():
    try:
        import psutil
        return psutil.virtual_memory().available
    except Exception:
        return float("inf")


def device_bytes_free():
    import torch
    free, _ = torch.cuda.mem_get_info(0)
    return free


def oracle_after(deck, V0, substeps):
    """The oracle's velocity after `substeps` substeps from V0 (ghost rows
    filled at t = 0)."""
    o = oracle.Sim(oracle.params_from_deck(deck))
    o.time = 0.0
    for c in range(3):
        o.field(c)[...] = V0[c]
        o.fill_ghosts(c)
    o.deltat = deck["deltat"]
    for k in range(substeps):
        o.substep(k % 3)
    V = np.stack([o.field(c).copy() for c in range(3)])
    t = o.time
    del o
    return V, t


def gpu_after(deck, V0, steps, precision):
    s = hst.Solver(dict(deck, precision=precision))
    s.time = 0.0
    s.set_velocity(V0)
    for _ in range(steps):
        s.timestep(deck["deltat"])
    V = s.velocity()
    t = s.time
    s.close()
    return V, t


def check_both(name, substeps=30):
    w = WORKLOADS[name]
    deck = dict(w["deck"])
    y = oracle.Sim(oracle.params_from_deck(dict(deck, nx=1, nz=1))).y()
    V0 = seeded_field(name, y)
    Vo, to = oracle_after(deck, V0, substeps)
    errs = {}
    for prec, tol in (("fp64", FP64_TOL), ("mixed", MIXED_TOL)):
        Vg, tg = gpu_after(deck, V0, substeps // 3, prec)
        assert abs(tg - to) <= 1e-15 * max(1.0, abs(to))
        errs[prec] = rel_l2(Vg, Vo)
        del Vg
    assert errs["fp64"] <= FP64_TOL, errs
    assert errs["mixed"] <= MIXED_TOL, errs
    return errs


def test_384x384x256_against_oracle():
    """The 384^2 x 256 workload (deck nx = 127, nz = 128, ny = 256), 30
    substeps: FP64 <= 1e-12 and mixed <= 1e-5 relative L2 against the
    oracle.  Runs the FP64 k_zinv/k_zfwd 384-point 16-points-a-thread plans and
    the 8-point x plan at 384 that the timed configuration uses."""
    print(check_both("c2"))


def test_768x768x512_against_oracle():
    """The 768^2 x 512 exact_shift workload ("512^3": deck nx = 255, nz = 256,
    ny = 512, Re 5000, dt 0.001), 30 substeps from the seeded field with
    k0 = 16: FP64 <= 1e-12 and mixed <= 1e-5 relative L2 against the oracle.
    The oracle needs about 23 GB of host memory and minutes of host time."""
    if host_bytes_available() < 48e9:
        pytest.skip("the oracle at 768^2 x 512 needs about 48 GB of free host memory")
    if device_bytes_free() < 40e9:
        pytest.skip("the 768^2 x 512 context needs about 30 GB of device memory")
    print(check_both("c3"))


def test_768x768x512_mixed_statistics_3000_substeps():
    """The mixed-precision form against the FP64 form over 3000 substeps of
    the 768^2 x 512 workload from the same seeded field: the time averages of
    the energy and the dissipation (hst_gpu_outstats, src/hst_stats.f90:136-285
    on the device, every 30 substeps) agree within 0.5 %.  About three
    minutes of device time."""
    if device_bytes_free() < 40e9:
        pytest.skip("the 768^2 x 512 context needs about 30 GB of device memory")
    w = WORKLOADS["c3"]
    deck = dict(w["deck"])
    y = oracle.Sim(oracle.params_from_deck(dict(deck, nx=1, nz=1))).y()
    V0 = seeded_field("c3", y)
    runs = {}
    for prec in ("fp64", "mixed"):
        s = hst.Solver(dict(deck, precision=prec))
        s.time = 0.0
        s.set_velocity(V0)
        e, d = [], []
        for _ in range(100):
            s.timesteps(10, deck["deltat"])
            st = s.outstats()
            e.append(st["energy"])
            d.append(st["diss"])
        assert all(math.isfinite(v) for v in e + d)
        runs[prec] = (float(np.mean(e)), float(np.mean(d)))
        s.close()
    (e64, d64), (emp, dmp) = runs["fp64"], runs["mixed"]
    print("energy", e64, emp, "dissipation", d64, dmp)
    assert abs(emp - e64) <= 5e-3 * abs(e64)
    assert abs(dmp - d64) <= 5e-3 * abs(d64)


@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("mixed", MIXED_TOL)])
@pytest.mark.parametrize("axis", ["x", "z"])
def test_768_plans_parity(prec, tol, axis):
    """Each 768-point direction on a narrow deck (nx = 255: 2 nxd = 768; nz =
    256: nzd = 768), 64 rows, with exact_shift and an oscillating S2 (the
    branches the 768^2 x 512 workload adds to the default path), 9 substeps
    against the oracle."""
    sizes = dict(nx=255, nz=32) if axis == "x" else dict(nx=31, nz=256)
    deck = c1_deck(ny=64, re=5000.0, deltat=0.001, exact_shift=True, s2_amplitude=0.5, s2_period=10.0, **sizes)
    y = oracle.Sim(oracle.params_from_deck(dict(deck, nx=1, nz=1))).y()
    V0 = hst.random_field(deck["nx"], deck["ny"], deck["nz"], 1.0, 1.0, deck["ly"], y, seed=5, k0=16.0, energy=0.1)
    s, o = make_pair(dict(deck, precision=prec), V0)
    assert (2 * s.nxd if axis == "x" else s.nzd) == 768
    Vg, Vo = run_pair(s, o, deck["deltat"], 3)
    s.close()
    err = rel_l2(Vg, Vo)
    assert err <= tol, err


@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("mixed", MIXED_TOL)])
@pytest.mark.parametrize("exact", [False, True])
def test_s2_edge_modes_parity(prec, tol, exact):
    """With a spanwise shear S2 and the reference's padding nzd = 3 nz (here
    nz = 32, nzd = 96) the retained modes iz = +-nz of the products alias the
    product modes -+2nz, so the products of the ghost rows are not the wrap
    images of the interior rows' (their phases differ): the ghost rows are
    transformed themselves, as the reference transforms every row.  30
    substeps with energy at the edge modes (k0 = 16) against the oracle."""
    deck = c1_deck(ny=64, re=5000.0, deltat=0.001, exact_shift=exact, s2_amplitude=0.5, s2_period=10.0, nx=31, nz=32)
    y = oracle.Sim(oracle.params_from_deck(dict(deck, nx=1, nz=1))).y()
    V0 = hst.random_field(deck["nx"], deck["ny"], deck["nz"], 1.0, 1.0, deck["ly"], y, seed=5, k0=16.0, energy=0.1)
    s, o = make_pair(dict(deck, precision=prec), V0)
    assert s.nzd == 3 * s.nz
    Vg, Vo = run_pair(s, o, deck["deltat"], 10)
    s.close()
    err = rel_l2(Vg, Vo)
    assert err <= tol, err


def test_nan_field_is_reported():
    """A field that has gone NaN must not read back a finite CFL number:
    hst_gpu_timestep returns HST_EFINITE (the reference's time loop would go
    on with a NaN dt, src/hst.f90:163-169).  The NaN is planted on the host."""
    deck = c1_deck()
    V0 = hst.random_field(deck["nx"], deck["ny"], deck["nz"], 1.0, 1.0, deck["ly"],
                          oracle.Sim(oracle.params_from_deck(deck)).y(), seed=2, k0=4.0, energy=0.1)
    s = hst.Solver(deck)
    s.set_velocity(V0)
    s.timestep(deck["deltat"])
    assert math.isfinite(s.cfl)
    V = V0.copy()
    V[1, 3, s.nz + 2, 10] = complex(float("nan"), 0.0)
    s.set_velocity(V)
    with pytest.raises(hst.HstError) as e:
        s.timestep(deck["deltat"])
    assert e.value.code == hst.EFINITE
    # an infinity as well
    V = V0.copy()
    V[0, 0, s.nz, 7] = complex(float("inf"), 0.0)
    s.set_velocity(V)
    with pytest.raises(hst.HstError) as e:
        s.compute_cfl()
    assert e.value.code == hst.EFINITE
    # the context stays usable: a finite field (and cleared carried terms,
    # which the failed steps left NaN) steps again
    s.set_velocity(V0)
    zero = np.zeros(s.shape, np.complex128)
    s.upload(hst.OLD1, zero)
    s.upload(hst.OLD2, zero)
    s.timestep(deck["deltat"])
    assert math.isfinite(s.cfl)
    s.close()


def test_restart_errors(tmp_path):
    """hst_gpu_read_restart refuses a truncated file and a file of another
    mesh with HST_EARG (restart_read's checks, src/hst_io.f90:69-178), and a
    missing file; the resident field is left as it was."""
    deck = c1_deck(nx=15, nz=16, ny=32)
    s = hst.Solver(deck)
    V0 = hst.random_field(deck["nx"], deck["ny"], deck["nz"], 1.0, 1.0, deck["ly"], s.y, seed=3, k0=4.0, energy=0.1)
    s.set_velocity(V0)
    good = tmp_path / "Dati.cart"
    s.write_restart(good)
    data = good.read_bytes()
    trunc = tmp_path / "truncated.cart"
    trunc.write_bytes(data[:len(data) - 4096])
    with pytest.raises(hst.HstError) as e:
        s.read_restart(trunc)
    assert e.value.code == hst.EARG and "truncated" in str(e.value)
    other = hst.Solver(c1_deck(nx=15, nz=16, ny=64))
    wrong = tmp_path / "other.cart"
    other.write_restart(wrong)
    other.close()
    with pytest.raises(hst.HstError) as e:
        s.read_restart(wrong)
    assert e.value.code == hst.EARG and "mesh" in str(e.value)
    with pytest.raises(hst.HstError) as e:
        s.read_restart(tmp_path / "absent.cart")
    assert e.value.code == hst.EARG
    assert rel_l2(s.velocity(), V0) <= 1e-15  # nothing was uploaded
    s.read_restart(good)
    assert rel_l2(s.velocity(), V0) <= 1e-15
    s.close()
