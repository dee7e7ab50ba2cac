"""Census of the flight loop's events on the self-consistent FinFET: how
many passes of the event loop end at a tetrahedron face, a cell face, a
scattering event (real or self-scattering) or the end of the step, per
particle-step, and how much work the rare shared tails do (get_state draws,
k-space walk steps).  It needs the engine built with the census compiled in
(one atomic per counted event, so never the timed build):

    make -C c-mc_electron_b200 EXTRA=-DMCB200_FLIGHT_EVENT_STATS=1 BUILD=_build_events LIB=libmcb200_events.so libmcb200_events.so
    MCB200_LIBRARY=c-mc_electron_b200/libmcb200_events.so python -m mcb200.flight_events [--fp64]

The deck is the throughput FinFET (decks.finfet at its defaults); 30 steps
from the seeded equilibrium, then 20 counted steps, each as density()
orders it (deposition, the Poisson solve every 10 steps, surface rates, the
carrier step).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import tempfile

import numpy as np

from . import FLIGHT_FP32, FLIGHT_FP64, NUM_COUNTERS, Deck, Engine, decks, lib

NAMES = {10: "tet_face", 11: "cell_face", 12: "scatter_event", 13: "step_end", 14: "get_state_draws",
         15: "walk_steps", 0: "phonon_real", 1: "impurity_real", 4: "loop_passes"}


def census(precision: int = FLIGHT_FP32, warm: int = 30, counted: int = 20, seed: int = 1) -> dict:
    with tempfile.TemporaryDirectory() as tmp:
        d = decks.finfet(tmp, total_step=warm + counted, heat_steps=0, stat_step=100000)
        deck = Deck(d["input"])
        root = Engine(max_particles=1, precision=precision)
        deck.prepare(root)
        n = int(deck.int_array("electron_num").sum() + deck.int_array("hole_num").sum())
        eng = Engine(max_particles=2 * n + 65536, precision=precision, like=root)
        deck.apply(eng)
        deck.seed(eng, seed)
        info = deck.info()
        eeff = deck.int_array("eeff_direction")
        deck.close()
    surf = dict(delta_m=0.4e-9, ail_m=1.5e-9, roughness=info["flag_surface_roughness"],
                phonon=info["flag_surface_phonon"])
    eng.deposit()
    eng.solve_poisson(1e-10, 20000)

    def run(s0, k):
        for s in range(s0, s0 + k):
            eng.deposit()
            if s % 10 == 0:
                eng.solve_poisson_async(1e-10, 20000)
            eng.surface_rates(eeff, **surf)
            eng.step(s, seed, info["dt"])

    run(0, warm)
    eng.sync()
    eng.reset_tallies()
    ps0 = eng.particle_steps()
    run(warm, counted)
    eng.sync()
    ps = eng.particle_steps() - ps0
    c = np.zeros(NUM_COUNTERS, dtype=np.uint64)
    eng._check(lib().mcb200_get_tallies(eng._ctx, c.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), None, None,
                                        None, None, None), "tallies")
    eng.close()
    root.close()
    return {"precision": "fp64" if precision == FLIGHT_FP64 else "fp32", "particle_steps": int(ps),
            "per_particle_step": {NAMES[i]: float(c[i]) / ps for i in sorted(NAMES)}}


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--fp64", action="store_true")
    a = ap.parse_args()
    print(json.dumps(census(FLIGHT_FP64 if a.fp64 else FLIGHT_FP32), indent=1))


if __name__ == "__main__":
    main()
