"""Batched stepping (mcb200_batch_*): simulations of uneven size -- two
frozen-field bulk boxes of different mesh, particle count and field, and
two self-consistent FinFETs (gate lengths 20 and 15 nm) with GENERATE /
CATCH contacts whose copies go through every generation of the copy
flights -- step together in one batched flight launch per step; in full
timesteps where a FinFET solves Poisson, the members not solving fly beside
the solve (overlap: a side launch plus a helper launch sharing its work
counter).  Each member must end bit-identical to a
twin engine stepped alone (mcb200_deposit / mcb200_solve_poisson /
mcb200_step) from the same state: every particle (matched by uid), every
tally and the potential.  Both flight precisions; transport steps with the
host's own density calls, and full timesteps run by the batch, with and
without CUDA graphs.
"""
import os
import tempfile

import numpy as np
import pytest

import mcb200
from mcb200 import decks
from mcb200.workloads import bulk_box_engine

pytestmark = pytest.mark.gpu

STEPS = 12
POISSON_EVERY = 4
BULK = [dict(particles=4000, seed=3, nx=10, ny=6, nz=6, field_v_per_m=1e6),
        dict(particles=24000, seed=4, nx=20, ny=10, nz=8, field_v_per_m=5e6)]


def finfet_engine(tmp, precision, like, lg_nm=20.0, vg=0.8):
    deck = mcb200.Deck(decks.finfet(tmp, electrons=20000, holes=3000, surface_scatter=False, compute_heat=False,
                                    lg_nm=lg_nm, vg=vg)["input"])
    eng = mcb200.Engine(table_dir=mcb200.DEFAULT_TABLE_DIR, kelvin=deck.info()["temperature"],
                        max_particles=1 << 20, precision=precision, like=like)
    deck.apply(eng)
    deck.seed(eng, 11)
    eng.deposit()
    eng.solve_poisson(1e-10, 20000)
    dt = deck.info()["dt"]
    deck.close()
    return eng, dt


def build(tmp, precision, like=None):
    """The four members; the first made from scratch unless `like` is given,
    the others alike.  Returns [(engine, dt, seed, self_consistent)]."""
    out = []
    for spec in BULK:
        eng, dt, _ = bulk_box_engine(spec["particles"], spec["seed"], 0, precision=precision,
                                     like=like if like is not None else (out[0][0] if out else None),
                                     **{k: v for k, v in spec.items() if k not in ("particles", "seed")})
        out.append((eng, dt, 100 + spec["seed"], False))
    eng, dt = finfet_engine(os.path.join(tmp, "a"), precision, out[0][0])
    out.append((eng, dt, 200, True))
    eng, dt = finfet_engine(os.path.join(tmp, "b"), precision, out[0][0], lg_nm=15.0, vg=0.5)
    out.append((eng, dt, 300, True))
    return out


def density(eng, step, sc):
    if sc:
        eng.deposit()
        if step % POISSON_EVERY == 0:
            eng.solve_poisson_async(1e-10, 20000)


def by_uid(eng):
    d = eng.download()
    order = np.argsort(d["uid"], kind="stable")
    return {k: v[order] for k, v in d.items()}


def same_tallies(a, b):
    for k in a:
        if isinstance(a[k], np.ndarray):
            assert np.array_equal(a[k], b[k]), k
        else:
            assert a[k] == b[k], k


@pytest.mark.parametrize("precision", [mcb200.FLIGHT_FP64, mcb200.FLIGHT_FP32])
def test_batch_matches_members_alone(precision):
    with tempfile.TemporaryDirectory() as t1, tempfile.TemporaryDirectory() as t2:
        alone = build(t1, precision)
        batched = build(t2, precision, like=alone[0][0])
    for step in range(STEPS):
        for eng, dt, seed, sc in alone:
            density(eng, step, sc)
            eng.step(step, seed, dt)
    batch = mcb200.Batch([(eng, dt, seed, 0) for eng, dt, seed, _ in batched])
    for step in range(STEPS):
        for eng, _, _, sc in batched:
            density(eng, step, sc)
        batch.step()
    batch.sync()
    info = batch.info()
    assert info["members"] == 4 and info["steps"] == STEPS and info["launches"] == STEPS * 6
    for (ea, *_), (eb, *_) in zip(alone, batched):
        a, b = by_uid(ea), by_uid(eb)
        assert a["uid"].size > 0
        for k in a:
            assert np.array_equal(a[k], b[k]), k
        same_tallies(ea.tallies(), eb.tallies())
    # the FinFET member made copies, so the copy flights did work
    assert batched[2][0].tallies()["generated"] > 0
    batch.close()
    for eng, *_ in batched + alone:
        eng.close()


@pytest.mark.parametrize("precision,graphs,overlap", [(mcb200.FLIGHT_FP64, False, True),
                                                      (mcb200.FLIGHT_FP64, True, True),
                                                      (mcb200.FLIGHT_FP32, True, True),
                                                      (mcb200.FLIGHT_FP64, True, False)])
def test_batch_run_matches_members_alone(precision, graphs, overlap):
    with tempfile.TemporaryDirectory() as t1, tempfile.TemporaryDirectory() as t2:
        alone = build(t1, precision)
        batched = build(t2, precision, like=alone[0][0])
    # members start at different step numbers: the FinFETs solve on different
    # steps (t = 3, 7, 11 and 2, 6, 10), each flying beside the other's solve
    first = [0, 3, 5, 2]
    for step in range(STEPS):
        for (eng, dt, seed, sc), f in zip(alone, first):
            density(eng, f + step, sc)
            eng.step(f + step, seed, dt)
    batch = mcb200.Batch([(eng, dict(dt=dt, seed=seed, first_step=f, self_consistent=int(sc),
                                      poisson_every=POISSON_EVERY))
                          for (eng, dt, seed, sc), f in zip(batched, first)])
    batch.use_graphs(graphs)
    batch.set_overlap(overlap)
    batch.run(STEPS // 2)
    batch.run(STEPS - STEPS // 2)
    batch.sync()
    info = batch.info()
    solving = 6  # steps with a solve: two more launches each (side flight and helper) with overlap
    assert info["steps"] == STEPS and info["launches"] == STEPS * 6 + (2 * solving if overlap else 0)
    if graphs:
        assert info["graph_captures"] >= 2 and info["graph_captures"] + info["graph_replays"] == STEPS
    for (ea, *_), (eb, *_) in zip(alone, batched):
        a, b = by_uid(ea), by_uid(eb)
        for k in a:
            assert np.array_equal(a[k], b[k]), k
        same_tallies(ea.tallies(), eb.tallies())
    for k in (2, 3):
        pa, pb = alone[k][0].array("potential"), batched[k][0].array("potential")
        assert np.array_equal(pa.view(np.uint64), pb.view(np.uint64))
        assert alone[k][0].poisson_stats() == batched[k][0].poisson_stats()
    batch.close()
    for eng, *_ in batched + alone:
        eng.close()


@pytest.mark.parametrize("precision", [mcb200.FLIGHT_FP64, mcb200.FLIGHT_FP32])
def test_paired_solves_match_members_alone(precision):
    """Two FinFETs on the same mesh (Vg 0.8 and 0.5) solving on the same
    steps share one cooperative launch per solve (pairing); with a bulk box
    flying beside the pair.  Potentials, solver statistics, particles and
    tallies must equal those of twins stepped alone."""
    def members(tmp, like=None):
        bulk, dt0, _ = bulk_box_engine(4000, 3, 0, precision=precision, like=like, nx=10, ny=6, nz=6,
                                       field_v_per_m=1e6)
        out = [(bulk, dt0, 103, False)]
        for name, vg, seed in (("a", 0.8, 200), ("b", 0.5, 300)):
            eng, dt = finfet_engine(os.path.join(tmp, name), precision, bulk, vg=vg)
            out.append((eng, dt, seed, True))
        return out

    with tempfile.TemporaryDirectory() as t1, tempfile.TemporaryDirectory() as t2:
        alone = members(t1)
        batched = members(t2, like=alone[0][0])
    first = [0, 1, 1]  # the FinFETs solve together on t = 3, 7, 11
    for step in range(STEPS):
        for (eng, dt, seed, sc), f in zip(alone, first):
            density(eng, f + step, sc)
            eng.step(f + step, seed, dt)
    batch = mcb200.Batch([(eng, dict(dt=dt, seed=seed, first_step=f, self_consistent=int(sc),
                                      poisson_every=POISSON_EVERY))
                          for (eng, dt, seed, sc), f in zip(batched, first)])
    batch.use_graphs(True)
    batch.set_pairing(True)
    batch.run(STEPS)
    batch.sync()
    # 3 solving steps, each: one paired solve launch, the side flight and its helper
    assert batch.info()["launches"] == STEPS * 6 + 3 * 3
    for (ea, *_), (eb, *_) in zip(alone, batched):
        a, b = by_uid(ea), by_uid(eb)
        for k in a:
            assert np.array_equal(a[k], b[k]), k
        same_tallies(ea.tallies(), eb.tallies())
    for k in (1, 2):
        pa, pb = alone[k][0].array("potential"), batched[k][0].array("potential")
        assert np.array_equal(pa.view(np.uint64), pb.view(np.uint64))
        assert alone[k][0].poisson_stats() == batched[k][0].poisson_stats()
    assert alone[1][0].poisson_stats() != alone[2][0].poisson_stats()  # two different systems
    batch.close()
    for eng, *_ in batched + alone:
        eng.close()


def test_batch_rejects_mixed_tables():
    a, dt, _ = bulk_box_engine(1000, 1, 0, nx=6, ny=5, nz=4)
    b, _, _ = bulk_box_engine(1000, 2, 0, nx=6, ny=5, nz=4)  # its own tables, not alike
    with pytest.raises(mcb200.EngineError):
        mcb200.Batch([(a, dt, 1, 0), (b, dt, 2, 0)])
    a.close()
    b.close()


@pytest.mark.parametrize("precision", [mcb200.FLIGHT_FP64, mcb200.FLIGHT_FP32])
def test_sort_bucket_width_leaves_results_unchanged(precision):
    """Members whose step sort groups 8 (FinFETs) or 4 (bulk boxes) cells per
    bucket (mcb200_set_sort_bucket) end bit-identical to twins sorted by
    cell, stepped alone: the order of the store changes, no result does.
    The batched flights copy the member table into shared memory here."""
    with tempfile.TemporaryDirectory() as t1, tempfile.TemporaryDirectory() as t2:
        alone = build(t1, precision)
        batched = build(t2, precision, like=alone[0][0])
    for eng, _, _, sc in batched:
        eng.set_sort_bucket(8 if sc else 4)
        assert eng.sort_bucket == (8 if sc else 4)
    with pytest.raises(mcb200.EngineError):
        batched[0][0].set_sort_bucket(3)
    assert batched[0][0].sort_bucket == 4
    first = [0, 3, 5, 2]
    for step in range(STEPS):
        for (eng, dt, seed, sc), f in zip(alone, first):
            density(eng, f + step, sc)
            eng.step(f + step, seed, dt)
    batch = mcb200.Batch([(eng, dict(dt=dt, seed=seed, first_step=f, self_consistent=int(sc),
                                      poisson_every=POISSON_EVERY))
                          for (eng, dt, seed, sc), f in zip(batched, first)])
    batch.use_graphs(True)
    batch.set_smem_table(True)  # the other tests read the member table in place
    batch.run(STEPS)
    batch.sync()
    for (ea, *_), (eb, *_) in zip(alone, batched):
        a, b = by_uid(ea), by_uid(eb)
        for k in a:
            assert np.array_equal(a[k], b[k]), k
        same_tallies(ea.tallies(), eb.tallies())
    for k in (2, 3):
        pa, pb = alone[k][0].array("potential"), batched[k][0].array("potential")
        assert np.array_equal(pa.view(np.uint64), pb.view(np.uint64))
    batch.close()
    for eng, *_ in batched + alone:
        eng.close()


def test_autotune_picks_a_sort_bucket():
    """The autotuner's three stages (launch shapes, overlap / pairing, sort
    buckets) end on a setting it timed, and the members keep its width."""
    with tempfile.TemporaryDirectory() as tmp:
        members = build(tmp, mcb200.FLIGHT_FP32)
    batch = mcb200.Batch([(eng, dict(dt=dt, seed=seed, first_step=0, self_consistent=int(sc),
                                      poisson_every=POISSON_EVERY)) for eng, dt, seed, sc in members])
    batch.use_graphs(True)
    t = batch.autotune(2)
    assert t["sort_bucket"] in (1, 2, 4, 8) and 16 <= t["candidates"] <= 20 and t["ms_per_step"] > 0
    assert all(eng.sort_bucket == t["sort_bucket"] for eng, *_ in members)
    batch.close()
    for eng, *_ in members:
        eng.close()


@pytest.mark.parametrize("precision", [mcb200.FLIGHT_FP64, mcb200.FLIGHT_FP32])
def test_solo_members_match_members_alone(precision):
    """Members above a particle count fly in launches of their own on their
    own streams (mcb200_batch_set_solo), the others in the batched launches,
    full timesteps replayed from CUDA graphs: every member ends bit-identical
    to its twin stepped alone."""
    with tempfile.TemporaryDirectory() as t1, tempfile.TemporaryDirectory() as t2:
        alone = build(t1, precision)
        batched = build(t2, precision, like=alone[0][0])
    first = [0, 3, 5, 2]
    for step in range(STEPS):
        for (eng, dt, seed, sc), f in zip(alone, first):
            density(eng, f + step, sc)
            eng.step(f + step, seed, dt)
    batch = mcb200.Batch([(eng, dict(dt=dt, seed=seed, first_step=f, self_consistent=int(sc),
                                      poisson_every=POISSON_EVERY))
                          for (eng, dt, seed, sc), f in zip(batched, first)])
    batch.use_graphs(True)
    n_solo = batch.set_solo(10000)  # the 24k bulk box and both FinFETs; the 4k box stays batched
    assert 1 <= n_solo < 4, n_solo
    batch.run(STEPS // 2)
    assert batch.set_solo(0) == 0  # the rest of the steps all batched
    batch.run(STEPS - STEPS // 2)
    batch.sync()
    for (ea, *_), (eb, *_) in zip(alone, batched):
        a, b = by_uid(ea), by_uid(eb)
        for k in a:
            assert np.array_equal(a[k], b[k]), k
        same_tallies(ea.tallies(), eb.tallies())
    for k in (2, 3):
        pa, pb = alone[k][0].array("potential"), batched[k][0].array("potential")
        assert np.array_equal(pa.view(np.uint64), pb.view(np.uint64))
    batch.close()
    for eng, *_ in batched + alone:
        eng.close()
