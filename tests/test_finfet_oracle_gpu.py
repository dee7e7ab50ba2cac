"""The bench's own self-consistent n-FinFET (mcb200.decks.finfet: 80x50x40
nonuniform mesh, 300k e- + 50k h+ requested, 511,200 carriers after the
per-cell minimum) through the reference's routines (oracle) and the engine.

* Deposition and Poisson: the engine deposits the reference's initial
  ensemble and solves the FinFET system (gate with work-function shift,
  source / drain / substrate contacts, SiO2 and vacuum) by multigrid CG to a
  1e-12 relative residual; its potential agrees with the reference's (the
  oracle solves by BiCGSTAB to 1e-14) to 1e-8 of its largest value, its
  fields to 1e-7 of theirs.
* Flight: ten FP64 transport steps on the reference's fields and surface
  rates -- phonon, impurity and surface scattering, SCATTOX, GENERATE /
  CATCH contacts and section tallies, electrons and holes -- particle by
  particle: cells, tetrahedra, wedges and carrier types bit-exact, kinematics
  to 1e-9; the event counters and contact tallies equal.
"""
import tempfile

import numpy as np
import pytest

import mcb200
from mcb200 import decks
from oracle_bridge import Oracle
from parity_cases import compare, device_engine_from_oracle, push_fields

pytestmark = pytest.mark.gpu

SEED = 3
STEPS = 10


@pytest.fixture(scope="module")
def finfet_pair():
    with tempfile.TemporaryDirectory() as tmp:
        d = decks.finfet(tmp, total_step=STEPS, heat_steps=0, stat_step=100000)
        orc = Oracle()
        orc.init(d["input"], seed=SEED)
    p0 = orc.particles()
    assert len(p0["x"]) == 511200
    orc.density_and_field()
    orc.surface_rates()
    flags = (mcb200.FLAG_SURFACE_SCATTER if orc.scalar("flag_surface_scatter") else 0) | \
        (mcb200.FLAG_SURFACE_IMPURITY if orc.scalar("flag_surface_impurity") else 0)
    assert flags & mcb200.FLAG_SURFACE_SCATTER
    eng = device_engine_from_oracle(orc, max_particles=2 * len(p0["x"]), flags=flags)
    eng.upload(p0)
    yield orc, eng, p0
    eng.close()


def test_finfet_poisson_matches_reference(finfet_pair):
    orc, eng, _ = finfet_pair
    eng.deposit()
    for ours, ref in (("cell_charge_e", "c_electron_charge"), ("cell_charge_h", "c_hole_charge"),
                      ("node_density", "p_par_charge")):
        a, b = eng.array(ours), orc.array(ref)
        scale = np.max(np.abs(b))
        assert np.max(np.abs(a - b)) <= 1e-12 * scale, (ours, np.max(np.abs(a - b)) / scale)
    its, res = eng.solve_poisson(rel_tol=1e-12, max_iter=50000)
    assert res <= 1e-12, (its, res)
    ref = orc.array("p_poisson_pot")
    assert np.max(np.abs(eng.array("potential") - ref)) <= 1e-8 * np.max(np.abs(ref))
    f = np.stack([orc.array("c_field_x"), orc.array("c_field_y"), orc.array("c_field_z")], axis=1)
    e = eng.array("efield").reshape(-1, 3)
    assert np.max(np.abs(e + f)) <= 1e-7 * np.max(np.abs(f))


def test_finfet_flight_matches_reference(finfet_pair):
    orc, eng, _ = finfet_pair
    push_fields(orc, eng)  # the reference's fields and screening density, frozen for the steps
    eng.set_surface_rates(orc.array("c_e_roughnessRate"), orc.array("c_e_surfPhononRate"),
                          orc.array("c_h_roughnessRate"), orc.array("c_h_surfPhononRate"))
    dt = orc.scalar("dt")
    orc.reset_tallies()
    eng.reset_tallies()
    for s in range(STEPS):
        orc.flight_step(s)
        eng.step(s, SEED, dt)
        r = compare(orc.particles(), eng.download())
        assert r["mismatch"] == 0, (s, r)
    t = eng.tallies()
    assert t["phonon"] == int(orc.scalar("phonon_scatter")) > 0
    assert t["impurity"] == int(orc.scalar("impurity_scatter")) > 0
    assert t["generated"] == int(orc.scalar("gen_par"))
    assert t["caught"] == int(orc.scalar("catch_par_num"))
    assert t["no_tet"] == 0 and t["too_many_events"] == 0
    ref = orc.contacts()[:, :5]
    got = t["contact"][: len(ref), :5]
    assert np.array_equal(ref[:, [0, 3]], got[:, [0, 3]])
    # charge / energy sums: int64 fixed point (2^-40 charge, 2^-32 kT per term) against FP64 sums
    assert np.allclose(got, ref, rtol=1e-9, atol=1e-9 * max(np.abs(ref).max(), 1e-300))
    for side in ("lcurrent", "rcurrent"):
        a = orc.array(side)
        assert np.allclose(t[side], a, rtol=1e-9, atol=1e-9 * max(np.abs(a).max(), 1e-300)), side
