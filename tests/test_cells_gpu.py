"""GPU parity of the per-cell kernels and of surface scattering.

* surface rates (GetSurfRoughnessPhononScRate) from the same fields and
  screening density: relative 1e-12 (pow may round an ulp apart);
* MultipleRefresh: the reference's own gen_new_par_mr driven per cell in uid
  order with the engine's per-(cell, carrier) streams; the resulting cell
  populations must be identical (same source particles, same order, same
  charges);
* flight with surface scattering on (roughness -> Diffuse, surface phonon
  events): discrete state bit-exact, kinematics to 1e-9.
"""
import tempfile

import numpy as np
import pytest

import mcb200
from mcb200 import decks
from oracle_bridge import ORACLE_TABLES, Oracle
from parity_cases import compare, engine_from_oracle

pytestmark = pytest.mark.gpu


def surface_bar(seed=5, electrons=3000, holes=600):
    with tempfile.TemporaryDirectory() as tmp:
        deck = decks.contact_bar(tmp, vd=0.5, surfaces=True, electrons=electrons, holes=holes)
        orc = Oracle()
        orc.init(deck["input"], seed=seed)
    orc.density_and_field()
    orc.surface_rates()
    return orc


def test_surface_rates():
    orc = surface_bar()
    eng = engine_from_oracle(orc, max_particles=1 << 14)
    eng.surface_rates(orc.array("c_EeffDirection").astype(np.int32),
                      roughness=int(orc.scalar("flag_surface_roughness")),
                      phonon=int(orc.scalar("flag_surface_phonon")))
    for ours, ref in (("e_rough", "c_e_roughnessRate"), ("e_phonon", "c_e_surfPhononRate"),
                      ("h_rough", "c_h_roughnessRate"), ("h_phonon", "c_h_surfPhononRate")):
        a, b = eng.array(ours), orc.array(ref)
        assert np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)) <= 1e-12, ours
    eng.close()


@pytest.mark.parametrize("preload", [False, True])
def test_multiple_refresh(preload):
    """MultipleRefresh against the oracle; preload: the targets uploaded
    beforehand (mcb200_set_refresh_targets) instead of by the refresh."""
    with tempfile.TemporaryDirectory() as tmp:
        deck = decks.bulk_box(tmp, nx=6, ny=5, nz=4, electrons=2000, holes=400)
        orc = Oracle()
        orc.init(deck["input"], seed=9)
    p = orc.particles()
    cells = 6 * 5 * 4
    cell = (p["j"] * 6 + p["i"]) * 4 + p["k"]
    ne = np.bincount(cell[p["type"] == 0], minlength=cells)
    nh = np.bincount(cell[p["type"] == 1], minlength=cells)
    # half the cells far from their target (resampled), half close (kept)
    rng = np.random.default_rng(3)
    far = rng.random(cells) < 0.5
    de = np.where(far, 3 * ne + 1, ne).astype(np.int32)
    dh = np.where(far, nh + 5, nh).astype(np.int32)
    orc.set_array("c_desired_electron_number", de)
    orc.set_array("c_desired_hole_number", dh)
    step = 49
    gen_ref = orc.multiple_refresh(step)
    after = orc.particles()
    eng = engine_from_oracle(orc, max_particles=1 << 14)
    eng.upload(p)
    if preload:
        eng.set_refresh_targets(de, dh)
    gen = eng.multiple_refresh(de, dh, step, seed=9)
    got = eng.download()
    assert gen == gen_ref
    assert len(got["x"]) == len(after["x"])
    for f in ("x", "y", "z", "kx", "ky", "kz", "energy", "charge", "i", "j", "k", "itet", "isym", "type", "uid"):
        assert np.array_equal(got[f], after[f]), f
    # resampled particles are new ones: no uid appears twice
    assert len(np.unique(got["uid"])) == len(got["uid"])
    eng.close()


def test_flight_with_surface_scattering():
    orc = surface_bar(seed=17, electrons=2500, holes=500)
    eng = engine_from_oracle(orc, max_particles=1 << 14, flags=mcb200.FLAG_SURFACE_SCATTER)
    eng.set_surface_rates(orc.array("c_e_roughnessRate"), orc.array("c_e_surfPhononRate"),
                          orc.array("c_h_roughnessRate"), orc.array("c_h_surfPhononRate"))
    eng.upload(orc.particles())
    dt = orc.scalar("dt")
    orc.reset_tallies()
    for s in range(3):
        orc.flight_step(s)
        eng.step(s, 17, dt)
        r = compare(orc.particles(), eng.download())
        assert r["mismatch"] == 0, (s, r)
    t = eng.tallies()
    assert t["phonon"] == int(orc.scalar("phonon_scatter"))
    eng.close()
