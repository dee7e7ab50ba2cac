"""Generates tests/golden/finfet_oracle_windows.json: the FinFET precision
protocol of mcb200.precision (run_finfet) run through the reference's own
routines (the CPU oracle, oracle/_ref/libref_oracle.so) -- TEST
INFRASTRUCTURE.  Needs the built oracle and the reference's tables
(oracle/_ref/input); takes about half an hour on one core.

Per step, as the reference's density() orders it: statistic(); the
deposition and Poisson solve (density_and_field) every
FINFET_POISSON_EVERY steps, else compute_cell_charge; the surface rates;
update_particle (the oracle's flight step); MultipleRefresh every
FINFET_MR_STEP steps.  flag_heat is on, so phonon events tally heat.  The
surface-roughness delta and correlation length are set to the deck's
0.4 nm and 1.5 nm (the reference's scaling() sets 0.1127 nm and 2 nm).
Window sums are read with set_stat_zero() between windows and turned into
observables by mcb200.precision.finfet_observables, the function the
engine's windows go through.

    python tests/golden/make_finfet_oracle.py [--seeds 1 2 3 4 5 6] [--jobs 6] [--out ...]

One run per seed, the runs in parallel processes; the fixture holds every
run's windows (statistics across independent seeds give honest standard
errors: windows of one run are correlated).
"""
import argparse
import json
import os
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "c-mc_electron_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import numpy as np  # noqa: E402

from mcb200 import decks, precision as P  # noqa: E402
from oracle_bridge import Oracle  # noqa: E402


def run(seed: int) -> dict:
    warmup, windows, wsteps = P.FINFET_WARMUP, P.FINFET_WINDOWS, P.FINFET_WINDOW_STEPS
    with tempfile.TemporaryDirectory() as tmp:
        d = decks.finfet(tmp, total_step=warmup + windows * wsteps, heat_steps=0, compute_heat=False,
                         mr_step=P.FINFET_MR_STEP)
        orc = Oracle()
        orc.init(d["input"], seed=seed)
    u = {k: orc.scalar(k) for k in ("spr0", "time0", "eV0", "curr0")}
    orc.set_scalar("SurfSc_delta", 0.4e-9 / u["spr0"])
    orc.set_scalar("SurfSc_ail", 1.5e-9 / u["spr0"])
    orc.set_scalar("flag_heat", 1)
    dt = orc.scalar("dt")
    nx, ny, nz, px, py, pz = orc.dims()
    orc.density_and_field()
    t0 = time.time()
    step = 0

    def advance(n):
        nonlocal step
        for _ in range(n):
            orc.statistic()
            if step % P.FINFET_POISSON_EVERY == 0:
                orc.density_and_field()
            else:
                orc.compute_cell_charge()
            orc.surface_rates()
            orc.flight_step(step)
            if step % P.FINFET_MR_STEP == P.FINFET_MR_STEP - 1:
                orc.multiple_refresh(step)
            step += 1

    advance(warmup)
    rows = []
    for w in range(windows):
        orc.set_stat_zero()
        advance(wsteps)
        nc = int(orc.scalar("num_contact"))
        win = {"contact": orc.contacts()[:nc].tolist(), "lcurrent": orc.array("lcurrent").tolist(),
               "rcurrent": orc.array("rcurrent").tolist(), "electron_q": float(orc.array("stat_chargeE").sum()),
               "electron_qvy": float(orc.array("stat_vyE").sum()),
               "electron_qe": float(orc.array("stat_energyE").sum()),
               "heat": float(orc.array("p_electron_heat").sum() + orc.array("p_hole_heat").sum())}
        rows.append(P.finfet_observables(win, u, dt, wsteps, ny))
        print(f"seed {seed} window {w}: {rows[-1]}  ({time.time() - t0:.0f} s)", flush=True)
    return {"seed": seed, "particles_end": len(orc.particles()["x"]), "windows": rows,
            "cpu_seconds": time.time() - t0}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--seeds", type=int, nargs="+", default=[1, 2, 3, 4, 5, 6])
    ap.add_argument("--jobs", type=int, default=6)
    ap.add_argument("--out", default=os.path.join(HERE, "finfet_oracle_windows.json"))
    a = ap.parse_args()
    import multiprocessing as mp

    with mp.get_context("spawn").Pool(min(a.jobs, len(a.seeds))) as pool:
        runs = pool.map(run, a.seeds)
    out = {"protocol": {"warmup": P.FINFET_WARMUP, "windows": P.FINFET_WINDOWS, "window_steps": P.FINFET_WINDOW_STEPS,
                        "poisson_every": P.FINFET_POISSON_EVERY, "mr_step": P.FINFET_MR_STEP},
           "runs": runs}
    with open(a.out, "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
