"""The engine's own deck reader against the reference's initialisation.

Every deck is read twice: by mcb200_deck_load / mcb200_deck_prepare (C++ in
the engine library, csrc/deck.cpp) and by the reference's initialize()
(oracle).  All per-cell arrays, node coordinates, widths, contacts, surfaces
and the compute_par_num carrier counts must be identical, bit for bit.
Decks: the contact bar (with and without surfaces), the bulk box, the
FinFET deck the engine is measured on, and -- where the reference tree is
present -- a copy of the reference's own finfet/ deck with its carrier
counts lowered so the oracle initialises quickly.
"""
import os
import shutil
import tempfile

import numpy as np
import pytest

import mcb200
from mcb200 import decks
from oracle_bridge import ORACLE_TABLES, Oracle
from parity_cases import action_bar, make_restart

REF_FINFET = os.path.join(os.environ.get("MCB200_REFERENCE", "/root/reference"), "finfet")


def _compare(input_path):
    deck = mcb200.Deck(input_path)
    eng = mcb200.Engine(table_dir=ORACLE_TABLES, kelvin=deck.info()["temperature"], device=-1)
    deck.prepare(eng)
    orc = Oracle()
    orc.init(input_path, seed=1)
    info = deck.info()
    cells = info["nx"] * info["ny"] * info["nz"]
    as_int = lambda a: np.asarray(a).astype(np.int64)
    pairs_int = [("material", "c_material"), ("attached_contact", "c_attached_contact"),
                 ("in_surf_region", "c_InSurfRegion"), ("motion_rule", "c_motion_rule"),
                 ("scatter_type", "c_scatter_type"), ("quantum_region", "c_quantumRegion"),
                 ("electron_num", "c_electron_num"), ("hole_num", "c_hole_num"),
                 ("refresh_electrons", "c_desired_electron_number"), ("refresh_holes", "c_desired_hole_number")]
    if info["flag_surface_scatter"]:
        pairs_int += [("nearest_surf", "c_nearestSurf"), ("eeff_direction", "c_EeffDirection")]
    for ours, ref in pairs_int:
        a, b = as_int(deck.int_array(ours)), as_int(orc.array(ref))
        assert a.shape == b.shape, (ours, a.shape, b.shape)
        assert np.array_equal(a, b), ours
    for ours, ref in [("donor", "c_donor"), ("acceptor", "c_acceptor"), ("volume", "c_volume"), ("da", "c_da"),
                      ("init_electron_charge", "c_init_electron_charge"), ("init_hole_charge", "c_init_hole_charge"),
                      ("lx", "lx"), ("ly", "ly"), ("lz", "lz"), ("dx", "dx"), ("dy", "dy"), ("dz", "dz")]:
        a, b = deck.double_array(ours), orc.array(ref)
        assert np.array_equal(a, b), ours
    assert len(deck.int_array("material")) == cells
    # contacts: count, planes, normalised Vapp and PhiMS
    vapp, phims, planes = orc.contact_info()
    assert info["n_contacts"] == len(vapp)
    assert np.array_equal(deck.double_array("contact_vapp"), vapp)
    assert np.array_equal(deck.double_array("contact_phims"), phims)
    assert np.array_equal(deck.int_array("contact_planes").reshape(-1, 7), planes)
    # surfaces
    n = info["n_surfaces"]
    assert n == int(orc.scalar("num_surface"))
    assert np.array_equal(deck.int_array("surface_dir"), orc.array("SurfaceDir")[:n].astype(np.int32))
    assert np.array_equal(deck.int_array("surface_type"), orc.array("SurfaceType")[:n].astype(np.int32))
    assert np.array_equal(deck.double_array("surface_pos"), orc.array("SurfacePosition")[:n])
    # run parameters
    assert info["dt"] == orc.scalar("dt")
    for key, ref in [("total_step", "total_step"), ("electron_number", "electron_number"),
                     ("hole_number", "hole_number"), ("stat_step", "stat_step"), ("mr_step", "mr_step"),
                     ("default_electrons", "default_electron_num"), ("default_holes", "default_hole_num")]:
        assert info[key] == int(orc.scalar(ref)), key
    # the initial ensemble's size is the sum of the per-cell counts
    assert int(deck.int_array("electron_num").sum() + deck.int_array("hole_num").sum()) == len(orc.particles()["x"])
    eng.close()
    deck.close()


def test_contact_bar_deck():
    with tempfile.TemporaryDirectory() as tmp:
        d = decks.contact_bar(tmp, vd=0.4, electrons=3000, holes=500)
        _compare(d["input"])


def test_action_bar_deck():
    """PERIOD / SCATTOX / CATCH / GENERATE / CATCHGATE / GENREF faces and
    attachcontact parse to the reference's cell arrays."""
    with tempfile.TemporaryDirectory() as tmp:
        d = action_bar(tmp)
        _compare(d["input"])
        orc = Oracle()
        orc.init(d["input"], seed=1)
        rules = set(orc.array("c_motion_rule").astype(int).tolist())
        contact = orc.array("c_attached_contact").astype(int)
    # every action of HitCell appears (PASS 1, REFLECT 2, SCATTOX 3, PERIOD 4, GENERATE 5, GENREF 6, CATCH 7, CATCHGATE 8)
    assert rules >= {1, 2, 3, 4, 5, 6, 7, 8}, rules
    assert set(contact.tolist()) == {0, 1, 2}


def test_contact_bar_with_surfaces_deck():
    with tempfile.TemporaryDirectory() as tmp:
        d = decks.contact_bar(tmp, vd=0.4, electrons=3000, holes=500, surfaces=True)
        _compare(d["input"])


def test_restart_deck():
    """Flag_restart: the restart file's counts replace the computed ones
    (contact cells included), as the reference's init_particle_data reads
    them; the refresh targets keep the computed counts."""
    with tempfile.TemporaryDirectory() as tmp:
        d = decks.contact_bar(tmp, vd=0.4, electrons=3000, holes=500)
        make_restart(d)
        _compare(d["input"])
        deck = mcb200.Deck(d["input"])
        assert deck.info()["flag_restart"] == 1 and deck.info()["restart_step"] == 7
        deck.close()


def test_restart_deck_errors():
    with tempfile.TemporaryDirectory() as tmp:
        d = decks.contact_bar(tmp, electrons=300)
        make_restart(d)
        path = os.path.join(tmp, "restart.txt")
        with open(path) as f:
            body = f.read().splitlines()
        with open(path, "w") as f:
            f.write("\n".join(body[:-1]) + "\n")  # no -1 line
        deck = mcb200.Deck(d["input"])
        eng = mcb200.Engine(table_dir=ORACLE_TABLES, kelvin=deck.info()["temperature"], device=-1)
        with pytest.raises(mcb200.EngineError, match="restart"):
            deck.prepare(eng)
        eng.close()
        deck.close()


def test_bulk_box_deck():
    with tempfile.TemporaryDirectory() as tmp:
        d = decks.bulk_box(tmp, nx=7, ny=5, nz=4, electrons=2000, holes=300)
        _compare(d["input"])


def test_finfet_deck():
    with tempfile.TemporaryDirectory() as tmp:
        d = decks.finfet(tmp, electrons=20000, holes=4000)
        _compare(d["input"])


@pytest.mark.skipif(not os.path.isdir(REF_FINFET), reason="reference tree not present")
def test_reference_finfet_deck():
    with tempfile.TemporaryDirectory() as tmp:
        for f in ("lgrid.txt", "ldg.txt"):
            shutil.copy(os.path.join(REF_FINFET, f), tmp)
        lines = open(os.path.join(REF_FINFET, "input.txt")).read().splitlines()
        out = []
        for line in lines:
            key = line.split("=")[0].strip()
            if key == "ElectronNumber":
                line = "ElectronNumber=20000"
            elif key == "HoleNumber":
                line = "HoleNumber=4000"
            out.append(line)
        with open(os.path.join(tmp, "input.txt"), "w") as f:
            f.write("\n".join(out) + "\n")
        _compare(os.path.join(tmp, "input.txt"))


def test_deck_errors():
    with tempfile.TemporaryDirectory() as tmp:
        d = decks.contact_bar(tmp)
        with open(d["device"]) as f:
            text = f.read()
        with open(d["device"], "w") as f:
            f.write(text.replace("region 0 40", "region 0 41", 1))  # off the 5 nm grid
        with pytest.raises(mcb200.EngineError, match="not on a grid line"):
            mcb200.Deck(d["input"])
        with open(d["device"], "w") as f:
            f.write(text.replace("end\n", ""))
        with pytest.raises(mcb200.EngineError, match="without `end`"):
            mcb200.Deck(d["input"])
    with pytest.raises(mcb200.EngineError, match="cannot open"):
        mcb200.Deck("/nonexistent/input.txt")
