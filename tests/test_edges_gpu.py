"""Edge cases of the carrier step on the GPU.

* an empty store: a step, a deposition, a Poisson solve, the statistics
  and a refresh of an empty store run and leave it empty, with nothing
  tallied and nothing flown;
* one particle (a ragged launch: one lane of one warp busy) flies exactly
  as the reference's particle_fly flies it, step after step, in both
  precisions' common discrete state (FP64 against the oracle);
* a store too small for the GENERATE copies of a step: the step keeps the
  store full, drops the excess copies, counts them, and the next call that
  reports a status returns MCB200_ERR_CAPACITY (the reference grows its
  lists without bound; a fixed device store must report instead);
* the pipelined tally readback returns the tallies as they were when the
  copy was enqueued, after later steps have run, and refuses an empty slot;
* sampled step timing (one step in k bracketed by events) counts the
  sampled steps' flights and every step's particles.
"""
import tempfile

import numpy as np
import pytest

import mcb200
from mcb200 import decks
from oracle_bridge import Oracle
from parity_cases import action_bar, compare, device_engine_from_oracle, engine_from_oracle, push_fields, set_uniform_field

pytestmark = pytest.mark.gpu


def _bar_oracle(tmp, seed):
    d = action_bar(tmp)
    orc = Oracle()
    orc.init(d["input"], seed=seed)
    return orc


@pytest.mark.parametrize("precision", [mcb200.FLIGHT_FP64, mcb200.FLIGHT_FP32])
def test_empty_store(precision):
    with tempfile.TemporaryDirectory() as tmp:
        orc = _bar_oracle(tmp, 3)
    eng = device_engine_from_oracle(orc, precision=precision)
    empty = {k: v[:0] for k, v in orc.particles().items()}
    eng.upload(empty)
    dt = orc.scalar("dt")
    eng.reset_tallies()
    eng.stat_begin(2)
    for s in range(2):
        eng.stat_accumulate()
        eng.deposit()
        its, res = eng.solve_poisson(1e-10, 20000)
        eng.step(s, 3, dt)
    assert eng.num_particles() == 0 and eng.particle_steps() == 0
    t = eng.tallies()
    assert t["generated"] == 0 and t["caught"] == 0 and t["events"] == 0
    assert not np.any(t["contact"]) and not np.any(t["lcurrent"]) and not np.any(t["rcurrent"])
    assert not np.any(eng.stat("electron_q")) and not np.any(eng.stat("cell_count"))
    assert not np.any(eng.array("cell_charge_e"))
    n = eng.mesh.ncells
    assert eng.multiple_refresh(np.ones(n, np.int32), np.ones(n, np.int32), 9, 3) == 0  # nothing to resample
    assert eng.num_particles() == 0
    eng.close()


def test_one_particle_matches_the_reference():
    with tempfile.TemporaryDirectory() as tmp:
        deck = decks.bulk_box(tmp, nx=8, ny=6, nz=6, electrons=200, holes=50)
        orc = Oracle()
        orc.init(deck["input"], seed=17, make_particles=True)
    set_uniform_field(orc, 5e6)
    orc.compute_cell_charge()
    p = orc.particles()
    one = {k: v[:1].copy() for k, v in p.items()}
    orc.set_particles(one, orc.scalar("dt"))
    eng = engine_from_oracle(orc, max_particles=4096)
    eng.upload(one)
    dt = orc.scalar("dt")
    events = 0
    for s in range(12):
        orc.flight_step(s)
        eng.step(s, 17, dt)
        r = compare(orc.particles(), eng.download())
        assert r["mismatch"] == 0, (s, r)
    t = eng.tallies()
    assert eng.num_particles() == 1 and eng.particle_steps() == 12
    assert t["events"] > 12  # it scattered, not only drifted
    assert t["phonon"] == int(orc.scalar("phonon_scatter"))
    eng.close()


def test_store_full_of_copies_reports_capacity():
    with tempfile.TemporaryDirectory() as tmp:
        orc = _bar_oracle(tmp, 21)
    orc.density_and_field()
    p = orc.particles()
    n = len(p["x"])
    eng = device_engine_from_oracle(orc, max_particles=n)  # no room for a single copy
    push_fields(orc, eng)
    eng.upload(p)
    dt = orc.scalar("dt")
    with pytest.raises(mcb200.EngineError, match="full"):
        for s in range(8):
            eng.step(s, 21, dt)
            eng.num_particles()  # reads the device counts; an overflow is reported by the next status
            eng.download()
    assert eng.num_particles() <= n  # the store never holds more than its capacity
    assert eng.tallies()["generated"] > 0
    eng.close()


def test_pipelined_tallies_are_snapshots():
    with tempfile.TemporaryDirectory() as tmp:
        orc = _bar_oracle(tmp, 5)
    orc.density_and_field()
    eng = device_engine_from_oracle(orc)
    push_fields(orc, eng)
    eng.upload(orc.particles())
    dt = orc.scalar("dt")
    with pytest.raises(mcb200.EngineError, match="nothing enqueued"):
        eng.tallies_collect(3)
    snaps = []
    for s in range(3):
        eng.step(s, 5, dt)
        eng.tallies_enqueue(s)
        snaps.append(eng.tallies()["contact"].copy())  # the same state, read synchronously
    eng.step(3, 5, dt)  # more work after the copies
    for s in range(3):
        assert np.array_equal(eng.tallies_collect(s), snaps[s]), s
    assert snaps[2][:, 0].sum() + snaps[2][:, 3].sum() > 0  # the bar generated or caught something
    eng.close()


def test_sampled_step_timing():
    with tempfile.TemporaryDirectory() as tmp:
        orc = _bar_oracle(tmp, 7)
    orc.density_and_field()
    eng = device_engine_from_oracle(orc)
    push_fields(orc, eng)
    eng.upload(orc.particles())
    dt = orc.scalar("dt")
    eng.set_timing(3)
    for s in range(7):
        eng.step(s, 7, dt)
    t = eng.timing()
    assert t["flight_launches"] == 3 and t["steps"] == 3  # steps 0, 3 and 6
    assert t["flight_ms"] > 0 and t["step_ms"] >= t["flight_ms"]
    assert t["particles_flown"] == eng.particle_steps()  # every step's particles
    eng.set_timing(1)
    eng.step(7, 7, dt)
    assert eng.timing()["flight_launches"] == 1
    eng.close()
