"""Serving bias-point requests (mcb200_server_*): continuous batching of
n-FinFET requests on one device.

* a cold-started request gives the same result alone and admitted together
  with other requests (of another gate length and bias): Ids, its standard
  error, windows, steps, particle-steps and final particle count are
  bit-identical, because every schedule counts the request's own steps and
  every particle draws from its own stream;
* a request of the same family as a converged one warm-starts from it (the
  nearest bias), and both stay as warm-start entries;
* the HBM budget holds a second request in the queue until the first one
  retires, and latency counts from the arrival time.
"""
import os
import tempfile

import pytest

import mcb200
from mcb200 import decks

pytestmark = pytest.mark.gpu

COLD = dict(max_steps=40, min_windows=1000, warm_windows_cold=0, warm_start=False, poisson_every=5)


def deck(tmp, name, vg, vd=0.7, lg=15.0, electrons=60000):
    return decks.finfet(os.path.join(tmp, name), electrons=electrons, holes=electrons // 6, vg=vg, vd=vd,
                        lg_nm=lg, min_per_cell=(1, 0), compute_heat=False)["input"]


def drive(server, rounds=200):
    out = []
    for _ in range(rounds):
        active, pending = server.round()
        out += server.results()
        if active == 0 and pending == 0:
            break
    return out


def by_id(results, rid):
    return next(r for r in results if r["id"] == rid)


@pytest.mark.parametrize("estimator", [mcb200.IDS_CONTACT, mcb200.IDS_INDUCED])
def test_same_result_alone_and_in_mix(estimator):
    """Also with Ids from the induced (Ramo-Shockley) current: its tally is
    summed in fixed point per step, so it does not depend on the store's
    order either."""
    cold = dict(COLD, ids_estimator=estimator)
    with tempfile.TemporaryDirectory() as tmp:
        a = deck(tmp, "a", 0.4)
        b = deck(tmp, "b", 0.8, lg=20.0)
        c = deck(tmp, "c", 0.0, vd=0.05)
        s1 = mcb200.Server(quantum_steps=10)
        ida = s1.submit(a, "lg15", (0.4, 0.7), seed=1, **cold)
        alone = by_id(drive(s1), ida)
        s1.close()
        s2 = mcb200.Server(quantum_steps=10)
        s2.submit(b, "lg20", (0.8, 0.7), seed=2, **cold)
        ida2 = s2.submit(a, "lg15", (0.4, 0.7), seed=1, **cold)
        s2.submit(c, "lg15", (0.0, 0.05), seed=3, **cold)
        res = drive(s2)
        mixed = by_id(res, ida2)
        assert len(res) == 3 and all(r["status"] == mcb200.SERVE_STEP_LIMIT for r in res)
        s2.close()
    assert alone["status"] == mcb200.SERVE_STEP_LIMIT and alone["steps"] == 40 and alone["windows"] == 4
    for k in ("ids", "ids_stderr", "windows", "steps", "particle_steps", "particles"):
        assert alone[k] == mixed[k], k
    assert alone["ids"] != 0.0


def test_warm_start_from_nearest_bias():
    with tempfile.TemporaryDirectory() as tmp:
        kw = dict(target_rel_err=1e9, min_windows=2, warm_windows_cold=0, warm_windows_warm=0, max_steps=200,
                  poisson_every=5)
        s = mcb200.Server(quantum_steps=10)
        ida = s.submit(deck(tmp, "a", 0.4), "lg15", (0.4, 0.7), seed=1, **kw)
        ra = by_id(drive(s), ida)
        assert ra["status"] == mcb200.SERVE_CONVERGED and ra["warm_from"] == 0
        far = s.submit(deck(tmp, "far", 0.8, lg=20.0), "lg20", (0.8, 0.7), seed=3, **kw)  # another family: cold
        idb = s.submit(deck(tmp, "b", 0.45), "lg15", (0.45, 0.7), seed=2, **kw)
        res = drive(s)
        assert by_id(res, idb)["warm_from"] == ida
        assert by_id(res, far)["warm_from"] == 0
        assert s.stats()["cached"] == 3
        s.close()


def test_warm_start_from_a_settled_running_request():
    """MCB200_WARM_SETTLED: with no converged bias of the family cached, a
    request starts from the nearest running request of its family that is
    past its transient windows; MCB200_WARM_CONVERGED waits for a converged
    one (and starts cold here), another family never donates."""
    with tempfile.TemporaryDirectory() as tmp:
        kw = dict(COLD, max_steps=30)
        s = mcb200.Server(quantum_steps=10)
        ida = s.submit(deck(tmp, "a", 0.4), "lg15", (0.4, 0.7), seed=1, **kw)
        s.round()  # a has one window: past its (empty) transient
        idb = s.submit(deck(tmp, "b", 0.45), "lg15", (0.45, 0.7), seed=2, **dict(kw, warm_start=mcb200.WARM_SETTLED))
        idc = s.submit(deck(tmp, "c", 0.5), "lg15", (0.5, 0.7), seed=3, **dict(kw, warm_start=mcb200.WARM_CONVERGED))
        far = s.submit(deck(tmp, "far", 0.8, lg=20.0), "lg20", (0.8, 0.7), seed=4,
                       **dict(kw, warm_start=mcb200.WARM_SETTLED))
        with pytest.raises(mcb200.EngineError):
            s.submit(deck(tmp, "bad", 0.4), "lg15", (0.4, 0.7), seed=5, **dict(kw, warm_start=3))
        res = drive(s)
        s.close()
    assert by_id(res, ida)["warm_from"] == 0
    assert by_id(res, idb)["warm_from"] == ida
    assert by_id(res, idc)["warm_from"] == 0
    assert by_id(res, far)["warm_from"] == 0
    assert all(r["status"] == mcb200.SERVE_STEP_LIMIT and r["steps"] == 30 for r in res)
    assert by_id(res, idb)["particles"] > 0 and by_id(res, idb)["ids"] != 0.0


def test_budget_queues_the_second_request():
    with tempfile.TemporaryDirectory() as tmp:
        a, a2 = deck(tmp, "a", 0.4), deck(tmp, "a2", 0.5)
        kw = dict(COLD, max_steps=20)
        s = mcb200.Server(quantum_steps=10)
        first = s.submit(a, "lg15", (0.4, 0.7), seed=1, **kw)
        one = by_id(drive(s), first)
        s.close()
        s = mcb200.Server(quantum_steps=10, hbm_budget_bytes=int(one["bytes"] * 1.5))
        t = s.now()
        i1 = s.submit(a, "lg15", (0.4, 0.7), seed=1, arrival_s=t, **kw)
        i2 = s.submit(a2, "lg15", (0.5, 0.7), seed=2, arrival_s=t, **kw)
        active, pending = s.round()
        assert (active, pending) == (1, 1)
        res = s.results() + drive(s)
        r1, r2 = by_id(res, i1), by_id(res, i2)
        assert r2["admit_s"] >= r1["done_s"]
        assert r2["done_s"] - r2["arrival_s"] > r1["done_s"] - r1["arrival_s"]
        s.close()
