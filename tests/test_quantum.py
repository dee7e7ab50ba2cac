"""Quantum-correction inputs on the host, against the reference run inside
the CPU oracle: the six phonon dispersion tables (init_deep,
src/ParticleUtils.cpp:750-806) bit-exact, and the deck's ep_parm /
quantum_start_step / quantumRegion as parsed."""
import os
import tempfile

import numpy as np
import pytest

import mcb200
from mcb200 import decks
from oracle_bridge import ORACLE_TABLES, Oracle

ROWS = [201, 201, 51, 51, 51, 51]
COLS = [120, 110, 160, 150, 160, 150]


@pytest.fixture(scope="module")
def oracle_box():
    with tempfile.TemporaryDirectory() as tmp:
        deck = decks.bulk_box(tmp, nx=4, ny=3, nz=3, electrons=100)
        orc = Oracle()
        orc.init(deck["input"], seed=1, make_particles=False)
    return orc


def test_dispersion_tables_bit_exact(oracle_box):
    eng = mcb200.Engine(table_dir=ORACLE_TABLES, kelvin=300.0, device=-1, max_particles=1)
    ours = eng.table("dispersion", np.float64)
    eng.close()
    assert ours.size == sum(r * c for r, c in zip(ROWS, COLS))
    off = 0
    for d, (r, c) in enumerate(zip(ROWS, COLS)):
        ref = oracle_box.dispersion(d, r, c)
        assert np.array_equal(ours[off:off + r * c].view(np.uint64), ref.view(np.uint64)), d
        off += r * c


def test_deck_quantum_settings():
    with tempfile.TemporaryDirectory() as tmp:
        d = decks.finfet(os.path.join(tmp, "q"), electrons=2000, holes=300, compute_heat=False,
                         quantum=(3.0, 0.5, 3.1, 7))
        deck = mcb200.Deck(d["input"])
        info = deck.info()
        region = deck.int_array("quantum_region")
        deck.close()
    assert info["flag_quantum_correction"] == 1 and info["quantum_start_step"] == 7
    # the gated fin (and the surface-scattering range, which the reference
    # also marks as quantum) is flagged
    assert 0 < region.sum() < region.size
