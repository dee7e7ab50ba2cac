"""Boundary actions, window statistics and the data/ writers against the
reference's own routines (oracle), on the action bar (tests/parity_cases.py):
PERIOD, SCATTOX without surface scattering (Diffuse), CATCH, GENERATE,
CATCHGATE and GENREF faces, two contacts, a self-consistent field.

* test_boundary_actions_match_oracle: flights through every action,
  particle by particle (discrete state bit-exact, kinematics to 1e-9), with
  the contact tallies (NumParGen, CharGen, EnergyGen, NumParCatch,
  CharCatch) and section currents equal -- and each action must have fired.
* test_statistics_and_outputs_match_oracle: a statistics window of three
  self-consistent steps.  The sums of statistic() (src/mcmodel.cpp:
  1167-1408: per node and carrier the CIC-weighted |q| v, |q| and |q| E,
  per cell the particle count, per node the potential) equal the
  reference's to 1e-9 of their largest entry (int64 fixed point against
  FP64 sums; the engine's CG and the oracle's BiCGSTAB potentials differ at
  1e-11).  Then mcb200_write_outputs and the reference's output_stat +
  current_scatter_info + output_for_restart (:971-1161, :756-842, :895-965)
  write the window's files: the same files, the same lines, every word
  equal and every number equal to the printed precision (the reference's
  default six significant digits: 2e-5 relative).
"""
import ctypes
import os
import re
import tempfile

import numpy as np
import pytest

import mcb200
from oracle_bridge import Oracle
from parity_cases import DISC_FIELDS, action_bar, compare, device_engine_from_oracle, push_fields

pytestmark = pytest.mark.gpu

SEED = 21


def _bar(tmp, seed=SEED):
    d = action_bar(tmp)
    orc = Oracle()
    orc.init(d["input"], seed=seed)
    return orc


def _contact_tallies(orc, eng):
    ref = orc.contacts()[:, :5]
    got = eng.tallies()["contact"][: len(ref), :5]
    return ref, got


def test_boundary_actions_match_oracle():
    with tempfile.TemporaryDirectory() as tmp:
        orc = _bar(tmp)
    orc.density_and_field()  # fields of the deposited initial ensemble (vd = 0.5 V)
    eng = device_engine_from_oracle(orc)
    push_fields(orc, eng)
    eng.upload(orc.particles())
    dt = orc.scalar("dt")
    orc.reset_tallies()
    eng.reset_tallies()
    for s in range(8):
        orc.flight_step(s)
        eng.step(s, SEED, dt)
        r = compare(orc.particles(), eng.download())
        assert r["mismatch"] == 0, (s, r)
    t = eng.tallies()
    assert t["generated"] == int(orc.scalar("gen_par"))
    assert t["caught"] == int(orc.scalar("catch_par_num"))
    ref, got = _contact_tallies(orc, eng)
    assert np.array_equal(ref[:, [0, 3]], got[:, [0, 3]])  # particle counts
    # charge / energy sums: int64 fixed point (2^-40 charge, 2^-32 kT per term) against FP64 sums
    assert np.allclose(got, ref, rtol=1e-9, atol=1e-9 * np.abs(ref).max())
    for side in ("lcurrent", "rcurrent"):
        a, b = orc.array(side), t[side]
        assert np.allclose(b, a, rtol=1e-9, atol=1e-9 * max(np.abs(a).max(), 1e-300)), side
    # every action fired: GENERATE (contact 0) and GENREF (contact 1) copies,
    # CATCH (contact 0) and CATCHGATE (contact 1) catches
    assert ref[0, 0] > 0 and ref[1, 0] > 0, ref
    assert ref[0, 3] > 0 and ref[1, 3] > 0, ref
    eng.close()


STAT_PAIRS = [("electron_qvx", "stat_vxE"), ("electron_qvy", "stat_vyE"), ("electron_qvz", "stat_vzE"),
              ("electron_q", "stat_chargeE"), ("electron_qe", "stat_energyE"),
              ("hole_qvx", "stat_vxH"), ("hole_qvy", "stat_vyH"), ("hole_qvz", "stat_vzH"),
              ("hole_q", "stat_chargeH"), ("hole_qe", "stat_energyH"),
              ("pot_sum", "stat_pot"), ("qc_pot_sum", "stat_qc_pot")]

NUMBER = re.compile(r"^[-+]?(\d+\.?\d*|\.\d+)([eE][-+]?\d+)?$")


def _compare_files(a_path, b_path, rel=2e-5):
    """Same lines and words; numbers equal to `rel` (six printed digits), or
    within 1e-9 of the file's largest number (a difference of two nearly
    equal sums: the reference's FP64 leaves rounding residue where the
    engine's fixed point gives exactly zero)."""
    a = open(a_path).read().split("\n")
    b = open(b_path).read().split("\n")
    assert len(a) == len(b), (os.path.basename(a_path), len(a), len(b))
    words = [w for line in a for w in line.replace("=", " = ").split() if NUMBER.match(w)]
    floor = 1e-9 * max([abs(float(w)) for w in words] + [1e-300])
    worst = 0.0
    for la, lb in zip(a, b):
        ta, tb = la.replace("=", " = ").split(), lb.replace("=", " = ").split()
        assert len(ta) == len(tb), (os.path.basename(a_path), la, lb)
        for wa, wb in zip(ta, tb):
            if NUMBER.match(wa) and NUMBER.match(wb):
                x, y = float(wa), float(wb)
                err = abs(x - y)
                assert err <= rel * max(abs(x), abs(y)) + floor, (os.path.basename(a_path), la, lb)
                worst = max(worst, err / max(abs(x), abs(y), 1e-300))
            else:
                assert wa == wb, (os.path.basename(a_path), la, lb)
    return worst


def test_statistics_and_outputs_match_oracle():
    window = 3
    with tempfile.TemporaryDirectory() as tmp:
        orc = _bar(tmp, seed=SEED + 1)
        eng = device_engine_from_oracle(orc)
        eng.upload(orc.particles())
        dt = orc.scalar("dt")
        lib = mcb200.lib()
        # a solved potential on both sides before the window (statistic() sums the last solve's)
        orc.density_and_field()
        eng.deposit()
        assert eng.solve_poisson(rel_tol=1e-12, max_iter=50000)[1] <= 1e-12
        orc.set_scalar("stat_step", window)
        orc.set_stat_zero()
        orc.reset_tallies()
        eng.reset_tallies()
        assert lib.mcb200_stat_begin(eng._ctx, window) == 0
        for s in range(window):
            # density(): statistic, deposition, Poisson + fields, then the flight
            orc.statistic()
            orc.density_and_field()
            orc.flight_step(s)
            assert lib.mcb200_stat_accumulate(eng._ctx) == 0
            eng.deposit()
            its, res = eng.solve_poisson(rel_tol=1e-12, max_iter=50000)
            assert res <= 1e-12
            eng.step(s, SEED + 1, dt)
            a, b = orc.particles(), eng.download()
            ia, ib = np.argsort(a["uid"]), np.argsort(b["uid"])
            assert np.array_equal(a["uid"][ia], b["uid"][ib]), s
            for f in DISC_FIELDS:
                assert np.array_equal(a[f][ia], b[f][ib]), (s, f)
        m = eng.mesh
        nodes, cells = m.nnodes, m.ncells
        dptr = lambda v: v.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        for ours, ref in STAT_PAIRS:
            got = np.zeros(nodes)
            assert lib.mcb200_stat_get(eng._ctx, ours.encode(), dptr(got), nodes) == 0, ours
            exp = orc.array(ref)
            assert exp.shape == got.shape, ours
            scale = max(np.abs(exp).max(), 1e-300)
            assert np.max(np.abs(got - exp)) <= 1e-9 * scale, (ours, np.max(np.abs(got - exp)) / scale)
        got = np.zeros(cells)
        assert lib.mcb200_stat_get(eng._ctx, b"cell_count", dptr(got), cells) == 0
        assert np.array_equal(got, orc.array("stat_enum"))

        # the window's files, written by both
        ref_dir, our_dir = os.path.join(tmp, "ref"), os.path.join(tmp, "ours")
        os.makedirs(ref_dir)
        orc.write_outputs(ref_dir, window - 1)
        lib.mcb200_write_outputs.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_double, ctypes.c_int, ctypes.c_int]
        ncont = int(orc.scalar("num_contact"))
        assert lib.mcb200_write_outputs(eng._ctx, os.path.join(our_dir, "data").encode(), window - 1, window, dt,
                                        ncont, 0) == 0
        names = sorted(os.listdir(os.path.join(ref_dir, "data")))
        assert names == sorted(os.listdir(os.path.join(our_dir, "data"))), names
        expected = {f"{p}{window - 1}" for p in ("section_current", "electron_num", "pot", "qc_pot", "Electron",
                                                 "Hole", "par_info_restart")} | {"current"}
        assert set(names) == expected, names
        for name in names:
            _compare_files(os.path.join(ref_dir, "data", name), os.path.join(our_dir, "data", name))
        text = open(os.path.join(our_dir, "data", "current")).read()
        assert re.search(r"NumParGen = [1-9]", text) and re.search(r"NumParCatch = [1-9]", text), text
    eng.close()
