"""Many independent simulations stepped as one batch (mcb200_batch_*).

build_mix(): a seeded mix of uneven simulations -- frozen-field bulk n-Si
boxes (mesh from 20^3 up to 80 x 40 x 50 cells, E_x uniform in 1-100 kV/cm)
and self-consistent n-FinFETs (gate length 15, 20 or 30 nm, Vg uniform in
0-0.8 V, Vd 0.7 V, surface scattering, Poisson every 10 steps,
MultipleRefresh every mr_step) -- with particle counts log-uniform between
two bounds.  Every engine shares one upload of the band tables
(mcb200_create_alike).  A FinFET holds at least one electron per silicon
cell (the deck's default_par_number), so its count is the larger of the
drawn one and that floor.

run_batched() / run_alone(): full timesteps of every member, batched (one
persistent flight launch per step over all members, steps replayed from
CUDA graphs) or one member after another (each member's own launches on its
own stream), with the MultipleRefresh of the FinFETs between chunks of
steps.
"""
from __future__ import annotations

import math
import os
import tempfile

import numpy as np

from . import FLIGHT_FP32, Batch, Deck, Engine, DEFAULT_TABLE_DIR
from . import decks
from .workloads import motion_rules, uniform_fields

POISSON_EVERY = 10


class Member:
    """One simulation: its engine, batch settings and (FinFET) refresh targets."""

    def __init__(self, kind, eng, cfg, desc, refresh=None, mr_step=0, surface=None):
        self.kind, self.eng, self.cfg, self.desc = kind, eng, cfg, desc
        self.refresh, self.mr_step, self.surface = refresh, mr_step, surface
        self.step = cfg["first_step"]


def bulk_member(like, nx, ny, nz, field_kv_cm, particles, seed, precision, table_dir=DEFAULT_TABLE_DIR):
    """A frozen-field bulk box (5 nm cells, 1e17 cm^-3 donors, REFLECT outside)
    with exactly `particles` electrons in cells drawn uniformly."""
    eng = Engine(table_dir=table_dir, max_particles=particles + particles // 8 + 4096, precision=precision,
                 like=like)
    u = eng.units()
    h = 5e-9 / u["spr0"]
    eng.set_mesh(np.arange(nx + 1) * h, np.arange(ny + 1) * h, np.arange(nz + 1) * h)
    cells = nx * ny * nz
    doping = 1e23 / u["conc0"]
    eng.set_cells(motion_rules(nx, ny, nz), np.full(cells, doping))
    eng.set_fields(*uniform_fields(eng, field_kv_cm * 1e5, 1e23))
    rng = np.random.default_rng(seed)
    cell_of = np.sort(rng.integers(0, cells, particles)).astype(np.int32)
    eng.seed(cell_of, np.full(particles, -doping * h ** 3 * cells / particles), 0, seed)
    cfg = dict(dt=1e-15 / u["time0"], seed=seed, first_step=0, self_consistent=0)
    return Member("bulk", eng, cfg, dict(mesh=[nx, ny, nz], field_kv_cm=field_kv_cm, particles=particles))


def finfet_member(like, tmp, lg_nm, vg, particles, seed, precision, first_step, table_dir=DEFAULT_TABLE_DIR,
                  mr_step=50):
    """A self-consistent FinFET deck (decks.finfet) ready to step: seeded,
    deposited, solved, surface rates set."""
    d = decks.finfet(tmp, electrons=particles, holes=max(particles // 6, 1), vg=vg, lg_nm=lg_nm,
                     min_per_cell=(1, 0), compute_heat=False, mr_step=mr_step)
    deck = Deck(d["input"])
    deck.prepare(like)  # units and intrinsic density from the shared tables
    carriers = int(deck.int_array("electron_num").sum() + deck.int_array("hole_num").sum())
    eng = Engine(table_dir=table_dir, max_particles=carriers + carriers // 2 + 8192, precision=precision, like=like)
    deck.apply(eng)
    deck.seed(eng, seed)
    eng.deposit()
    eng.solve_poisson(1e-10, 20000)
    info = deck.info()
    eeff = deck.int_array("eeff_direction")
    surface = (eeff, dict(delta_m=0.4e-9, ail_m=1.5e-9, roughness=info["flag_surface_roughness"],
                          phonon=info["flag_surface_phonon"]))
    eng.surface_rates(surface[0], **surface[1])
    refresh = (deck.int_array("refresh_electrons"), deck.int_array("refresh_holes"))
    eng.set_refresh_targets(*refresh)  # not at the first refresh, inside a running batch
    cfg = dict(dt=info["dt"], seed=seed, first_step=first_step, self_consistent=1, poisson_every=POISSON_EVERY,
               surface_rates=1)
    deck.close()
    return Member("finfet", eng, cfg, dict(lg_nm=lg_nm, vg=vg, particles=carriers, drawn=particles), refresh,
                  info["mr_step"] if info["flag_multiple_refresh"] else 0, surface)


def build_mix(n=64, seed=4, precision=FLIGHT_FP32, n_min=5000, n_max=500000, table_dir=DEFAULT_TABLE_DIR,
              finfet_fraction=0.5):
    """The seeded mix; returns [Member] (the first member's engine owns the tables)."""
    rng = np.random.default_rng(seed)
    kinds = np.array(["finfet"] * int(round(n * finfet_fraction)) + ["bulk"] * (n - int(round(n * finfet_fraction))))
    rng.shuffle(kinds)
    counts = np.exp(rng.uniform(math.log(n_min), math.log(n_max), n)).astype(int)
    root = Engine(table_dir=table_dir, max_particles=1, precision=precision)
    members = []
    with tempfile.TemporaryDirectory() as tmp:
        for i in range(n):
            if kinds[i] == "bulk":
                m = bulk_member(root, int(rng.integers(20, 81)), int(rng.integers(20, 41)), int(rng.integers(20, 51)),
                                float(rng.uniform(1.0, 100.0)), int(counts[i]), 1000 + i, precision, table_dir)
            else:
                m = finfet_member(root, os.path.join(tmp, f"ff{i}"), float(rng.choice([15.0, 20.0, 30.0])),
                                  float(rng.uniform(0.0, 0.8)), int(counts[i]), 1000 + i, precision,
                                  int(rng.integers(0, POISSON_EVERY)), table_dir)
            members.append(m)
    return members, root


def particle_steps(members) -> int:
    return sum(m.eng.particle_steps() for m in members)


def refresh_due(members, k):
    """MultipleRefresh of the FinFETs whose refresh step (the reference's
    step % mr_step == mr_step - 1) fell in the last k steps; it runs after
    them, up to k - 1 steps late."""
    for m in members:
        if m.kind == "finfet" and m.mr_step:
            hits = [s for s in range(m.step - k, m.step) if s % m.mr_step == m.mr_step - 1]
            if hits:
                m.eng.multiple_refresh(m.refresh[0], m.refresh[1], hits[-1], m.cfg["seed"], wait=False)


def run_batched(batch: Batch, members, steps: int, chunk: int = 10):
    """`steps` full timesteps of every member through the batch, the FinFETs'
    refreshes between chunks."""
    done = 0
    while done < steps:
        k = min(chunk, steps - done)
        batch.run(k)
        for m in members:
            m.step += k
        done += k
        refresh_due(members, k)


def run_alone(members, steps: int, chunk: int = 10):
    """The same timesteps, each member with its own launches on its own
    stream (mcb200_deposit / mcb200_solve_poisson / mcb200_surface_rates /
    mcb200_step): no batching."""
    done = 0
    while done < steps:
        k = min(chunk, steps - done)
        for _ in range(k):
            for m in members:
                e, c = m.eng, m.cfg
                if c["self_consistent"]:
                    e.deposit()
                    if m.step % c["poisson_every"] == 0:
                        e.solve_poisson_async(1e-10, 20000)
                    if m.surface is not None:
                        e.surface_rates(m.surface[0], **m.surface[1])
                e.step(m.step, c["seed"], c["dt"])
                m.step += 1
        done += k
        refresh_due(members, k)
