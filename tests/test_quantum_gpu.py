"""GPU parity of the quantum correction against the reference run inside
the CPU oracle.

* Flights with Flag_QuantumCorrection: the LO / TO / LA phonon events take
  their final energy from the dispersion tables (FEK*,
  src/ElectronPhononScatter.cpp:152-167, 633-1022).  Discrete state must
  match exactly and the kinematics to parity_cases.REL_TOL, as for the
  plain flight.
* The effective potential of an n-FinFET's quantum region
  (quantumPotential, src/mcmodel.cpp:2337-2403) from the oracle's own
  Poisson potential: to 1e-12 of the potential's range (CUDA's erf and
  glibc's may round an ulp apart), and the two carriers' fields from the
  plain and the corrected potential (compute_field, :2240-2262).
* A short self-consistent run of that deck through mcb200_run_deck with the
  correction switched on at quantum_start_step.
"""
import os
import tempfile

import numpy as np
import pytest

import mcb200
from mcb200 import decks
from oracle_bridge import ORACLE_TABLES, Oracle
from parity_cases import run_bulk_parity

pytestmark = pytest.mark.gpu

QC = (3.0, 0.5, 3.1, 0)  # window 3 theta, theta 0.5 nm, 3.1 V oxide barrier, on from step 0


@pytest.mark.parametrize("field", [1e6, 2e7])
def test_quantum_flight_matches_reference(field):
    r = run_bulk_parity(n_particles=1200, steps=4, seed=7, field_v_per_m=field, quantum=True)
    print(r)
    assert r["mismatch"] == 0, r
    assert r["phonon_engine"] == r["phonon_oracle"] > 0
    assert r["impurity_engine"] == r["impurity_oracle"]
    # the dispersion tables changed final energies: the same seed without
    # the correction ends elsewhere
    plain = run_bulk_parity(n_particles=1200, steps=4, seed=7, field_v_per_m=field)
    assert plain["mismatch"] == 0
    assert plain["energy_sum"] != r["energy_sum"]


def test_effective_potential_matches_reference():
    with tempfile.TemporaryDirectory() as tmp:
        d = decks.finfet(os.path.join(tmp, "q"), electrons=20000, holes=3000, surface_scatter=False,
                         compute_heat=False, quantum=QC)
        orc = Oracle()
        orc.init(d["input"], seed=3, make_particles=True)
        orc.init_quantum()
        orc.density_and_field()  # Poisson, then the correction (step 0 >= quantum_start_step 0)
        deck = mcb200.Deck(d["input"])
        eng = mcb200.Engine(table_dir=ORACLE_TABLES, kelvin=deck.info()["temperature"], max_particles=1 << 16)
        deck.apply(eng)
        deck.close()
    raw, corrected = orc.array("p_poisson_pot_saved"), orc.array("p_poisson_pot")
    region = raw != corrected
    assert region.sum() > 1000  # the quantum region's nodes moved
    ours = eng.quantum_potential(raw)
    scale = np.max(np.abs(corrected))
    assert np.max(np.abs(ours - corrected)) <= 1e-12 * scale, np.max(np.abs(ours - corrected)) / scale
    assert np.array_equal(ours[~region], raw[~region])
    eng.set_potentials(raw, corrected)
    e, h = eng.array("efield").reshape(-1, 3), eng.array("hfield").reshape(-1, 3)
    fe = -np.stack([orc.array("c_field_x"), orc.array("c_field_y"), orc.array("c_field_z")], axis=1)
    fh = np.stack([orc.array("c_h_field_x"), orc.array("c_h_field_y"), orc.array("c_h_field_z")], axis=1)
    for ours_f, ref_f in ((e, fe), (h, fh)):
        assert np.max(np.abs(ours_f - ref_f)) <= 1e-12 * np.max(np.abs(ref_f))
    assert not np.allclose(fe, -fh)  # electrons and holes feel different fields
    eng.close()


def test_run_deck_with_quantum_correction():
    """Six self-consistent steps, the correction on from step 2, outputs
    every 3 steps: the second window's mean electron potential (qc_pot)
    differs from the Poisson potential's (pot) on the quantum nodes only."""
    with tempfile.TemporaryDirectory() as tmp:
        d = decks.finfet(os.path.join(tmp, "q"), electrons=20000, holes=3000, compute_heat=False, stat_step=3,
                         quantum=(3.0, 0.5, 3.1, 2))
        data = os.path.join(tmp, "data")
        rep = mcb200.run_deck(d["input"], data_dir=data, table_dir=ORACLE_TABLES, max_steps=6, max_heat_steps=0,
                              poisson_every=1)
        names = sorted(os.listdir(data))
        pot_files = [n for n in names if n.startswith("pot")]
        qc_files = [n for n in names if n.startswith("qc_pot")]
        assert len(pot_files) == 2 and len(qc_files) == 2, names
        pot = np.loadtxt(os.path.join(data, sorted(pot_files)[-1]))
        qc = np.loadtxt(os.path.join(data, sorted(qc_files)[-1]))
    assert rep["steps_done"] == 6
    assert np.array_equal(pot[:, :3], qc[:, :3])
    moved = pot[:, 3] != qc[:, 3]
    assert 0 < moved.sum() < len(moved)
