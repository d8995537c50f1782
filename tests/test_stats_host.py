"""The host half of the spectra (spectrum_write's running average,
src/hst_stats.f90:110-134) on the oracle's sums: no GPU needed."""
import numpy as np

import oracle
from homogenenousshearturbulence_b200 import hst
from tests.gpu_util import c1_deck, seeded_field


def test_column_spectrum_adds_up_to_the_energy(tmp_path):
    """The averaged column energies of ColumnSpectrum sum to the box energy
    q2/2 that outstats reports (the (0,0) column about its box mean), and the
    written file has one line per column."""
    deck = c1_deck(nx=15, nz=16, ny=32)
    o = oracle.Sim(oracle.params_from_deck(deck))
    V0 = seeded_field(deck, seed=9, k0=4.0, energy=0.1)
    # a mean flow in the (0,0) column, so that the box-mean correction matters
    V0[0, 0, deck["nz"], 2:-2] += 0.3 + 0.1 * np.sin(o.y()[2:-2])
    for c in range(3):
        o.field(c)[...] = V0[c]
        o.fill_ghosts(c)
    spec = hst.ColumnSpectrum(o.dyl())
    energies = []
    for _ in range(3):
        o.deltat = deck["deltat"]
        o.timestep()
        sums, exz = o.outstats_sums()
        spec.add(dict(zip(hst.Solver.SUM_NAMES, sums)), exz)
        energies.append(o.outstats()["energy"])
    E = spec.energies()
    ly = deck["ly"]
    assert abs(E.sum() / ly - np.mean(energies)) <= 1e-12 * np.mean(energies)
    path = tmp_path / "spectrum.dat"
    spec.write(path, o.time, deck["alfa0"], deck["beta0"])
    lines = path.read_text().splitlines()
    assert len(lines) == 1 + (deck["nx"] + 1) * (2 * deck["nz"] + 1)
    assert spec.nacc == 0


def test_oracle_sums_agree_with_its_outstats():
    """The oracle's 16 sums reproduce its own outstats box averages."""
    deck = c1_deck(nx=15, nz=16, ny=32, damp_kpar=3.0, damp_kperp=2.0, damp_rate=0.5, damp_edge=0.3)
    o = oracle.Sim(oracle.params_from_deck(deck))
    V0 = seeded_field(deck, seed=2, k0=4.0, energy=0.1)
    for c in range(3):
        o.field(c)[...] = V0[c]
        o.fill_ghosts(c)
    o.deltat = deck["deltat"]
    o.timestep()
    sums, _ = o.outstats_sums()
    st = o.outstats()
    ly_w = float(np.sum(o.dyl()))
    uu = sums[2] - sums[7] ** 2 / ly_w
    ww = sums[4] - sums[8] ** 2 / ly_w
    assert abs(0.5 * (uu + sums[3] + ww) / deck["ly"] - st["energy"]) <= 1e-13 * st["energy"]
    assert abs(sums[0] / deck["re"] / deck["ly"] - st["diss"]) <= 1e-13 * st["diss"]
    assert sums[9] == 0.0 and sums[11] == 0.0
    assert abs(sums[12] - sums[0]) <= 1e-13 * sums[0]
    assert sums[15] > 0 and sums[13] > 0 and sums[14] > 0
