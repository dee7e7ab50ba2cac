"""FP32-flight error report: each ensemble observable of the bulk n-Si
velocity-field sweep (the frozen-field bulk box, 1 / 3 / 10 / 30 / 100 kV/cm)
from FP32 flight against the all-FP64 run (the FP64 path is bit-exact with
the reference's routines, so it stands for the CPU oracle too).

The box is the bulk workload's (N_D = 1e17 cm^-3, 300 K, dt = 1 fs, 5 nm
cells, REFLECT on every face) stretched to 1 um along the field (200 x 10 x
10 cells) so that within the 0.8 ps measured few electrons reach the far
wall.  Per field, precision and seed: warm-up steps, then `blocks` windows
of `block_steps` steps, each averaged with the window statistics
(statistic(), src/mcmodel.cpp:1167-1408): drift velocity
<v_x> = sum |q| v_x / sum |q| (m/s), mean energy sum |q| E / sum |q| (eV);
from the store at the end: valley occupation (isym / 8); from the tallies:
real phonon and impurity events per particle-step.

Errors are statistics over independent runs (seeds): a run's observable is
its time average, the standard error of a precision's mean is the spread of
its runs over sqrt(runs), and a difference is judged in units of the
combined standard error against the Student-t quantile of the 3-sigma
(99.73 %) level for its degrees of freedom.  Windows of one run are not
independent (the ensemble's mean energy and velocity relax over ~0.1-1 ps,
longer than a window), so batch means over them understate the error.

The FinFET half (finfet_report) runs the throughput FinFET the same way in
both precisions and compares both with the reference's own routines run
through the same protocol (tests/golden/finfet_oracle_windows.json).

    python -m mcb200.precision [--electrons 100000] [--seeds 8] [--json out.json]
    python -m mcb200.precision --finfet [--finfet-seeds 6] \
        [--oracle-runs tests/golden/finfet_oracle_windows.json] [--json out.json]
"""
from __future__ import annotations

import argparse
import ctypes
import json

import numpy as np

from . import FLIGHT_FP32, FLIGHT_FP64, lib
from .workloads import bulk_box_engine

FIELDS_KV_CM = (1.0, 3.0, 10.0, 30.0, 100.0)


def _stat(eng, name: str, n: int) -> np.ndarray:
    out = np.zeros(n)
    eng._check(lib().mcb200_stat_get(eng._ctx, name.encode(), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                     n), f"mcb200_stat_get {name}")
    return out


SWEEP_BOX = dict(nx=200, ny=10, nz=10)


def run_field(field_kv_cm: float, precision: int, electrons: int = 100000, warmup: int = 300, blocks: int = 5,
              block_steps: int = 100, seed: int = 11, device: int = 0) -> dict:
    eng, dt, _ = bulk_box_engine(electrons, seed, device, precision=precision, field_v_per_m=field_kv_cm * 1e5,
                                 **SWEEP_BOX)
    u = eng.units()
    velo0 = u["spr0"] / u["time0"]
    nodes = (eng.mesh.nx + 1) * (eng.mesh.ny + 1) * (eng.mesh.nz + 1)
    step = 0
    for _ in range(warmup):
        eng.step(step, seed, dt)
        step += 1
    eng.reset_tallies()
    flown = 0
    v_blocks, e_blocks = [], []
    for _ in range(blocks):
        eng._check(lib().mcb200_stat_begin(eng._ctx, block_steps), "mcb200_stat_begin")
        for _ in range(block_steps):
            eng._check(lib().mcb200_stat_accumulate(eng._ctx), "mcb200_stat_accumulate")
            n = eng.num_particles()
            eng.step(step, seed, dt)
            flown += n
            step += 1
        q = _stat(eng, "electron_q", nodes).sum()
        v_blocks.append(_stat(eng, "electron_qvx", nodes).sum() / q * velo0)
        e_blocks.append(_stat(eng, "electron_qe", nodes).sum() / q * u["eV0"])
    t = eng.tallies()
    p = eng.download()
    eng.close()
    valley = np.bincount(p["isym"] // 8, minlength=6) / len(p["isym"])
    vb, eb = np.array(v_blocks), np.array(e_blocks)
    return {
        "field_kv_cm": field_kv_cm, "electrons": len(p["isym"]),
        "drift_velocity_m_s": float(vb.mean()), "drift_velocity_se": float(vb.std(ddof=1) / np.sqrt(len(vb))),
        "mean_energy_ev": float(eb.mean()), "mean_energy_se": float(eb.std(ddof=1) / np.sqrt(len(eb))),
        "valley": valley.tolist(), "valley_se": np.sqrt(valley * (1 - valley) / len(p["isym"])).tolist(),
        "phonon_per_particle_step": t["phonon"] / flown, "phonon_se": np.sqrt(t["phonon"]) / flown,
        "impurity_per_particle_step": t["impurity"] / flown, "impurity_se": np.sqrt(t["impurity"]) / flown,
        "caught": t["caught"], "zero_time": t["zero_time"],
    }


def three_sigma_limit(dof: float) -> float:
    """The two-sided 99.73 % quantile (3 sigma for a normal variable) of
    Student's t with `dof` degrees of freedom."""
    from scipy.stats import t

    return float(t.ppf(0.99865, max(dof, 1.0)))


def compare_samples(ref, test) -> dict:
    """Mean of `test` against mean of `ref` (each a list of independent run
    values): relative error, the difference in combined standard errors, and
    the 3-sigma-level limit for the Welch degrees of freedom."""
    a, b = np.asarray(ref, dtype=float), np.asarray(test, dtype=float)
    va, vb = a.var(ddof=1) / len(a), b.var(ddof=1) / len(b)
    se = float(np.sqrt(va + vb))
    dof = (va + vb) ** 2 / (va ** 2 / (len(a) - 1) + vb ** 2 / (len(b) - 1)) if va + vb > 0 else 1e9
    d = float(b.mean() - a.mean())
    return {"ref": float(a.mean()), "test": float(b.mean()), "rel_error": d / abs(a.mean()) if a.mean() else 0.0,
            "sigmas": d / se if se > 0 else 0.0, "se": se, "dof": float(dof), "limit": three_sigma_limit(dof)}


SWEEP_KEYS = ("drift_velocity_m_s", "mean_energy_ev", "phonon_per_particle_step", "impurity_per_particle_step")


def compare(fp64_runs: list, fp32_runs: list) -> dict:
    """Every FP32 observable against FP64, over independent runs."""
    out = {key: compare_samples([r[key] for r in fp64_runs], [r[key] for r in fp32_runs]) for key in SWEEP_KEYS}
    va = np.array([r["valley"] for r in fp64_runs])
    vb = np.array([r["valley"] for r in fp32_runs])
    valleys = [compare_samples(va[:, v], vb[:, v]) for v in range(va.shape[1])]
    out["valley_max_sigmas"] = float(max(abs(c["sigmas"]) / c["limit"] * 3.0 for c in valleys))
    out["valley_max_abs_error"] = float(np.max(np.abs(vb.mean(0) - va.mean(0))))
    return out


def sweep(electrons: int = 100000, warmup: int = 300, blocks: int = 5, block_steps: int = 100,
          fields=FIELDS_KV_CM, seeds: int = 8, device: int = 0) -> list:
    rows = []
    for f in fields:
        r64 = [run_field(f, FLIGHT_FP64, electrons, warmup, blocks, block_steps, seed=11 + k, device=device)
               for k in range(seeds)]
        r32 = [run_field(f, FLIGHT_FP32, electrons, warmup, blocks, block_steps, seed=11 + k, device=device)
               for k in range(seeds)]
        rows.append({"field_kv_cm": f, "fp64": r64, "fp32": r32, "error": compare(r64, r32)})
    return rows


# ---------------------------------------------------------------- FinFET
# The self-consistent n-FinFET of the throughput workload (decks.finfet at
# its defaults: 511,200 carriers, Vd 0.7 V, Vg 0.8 V, dt 0.2 fs, surface
# scattering), run from its equilibrium start through FINFET_WARMUP steps,
# then FINFET_WINDOWS windows of FINFET_WINDOW_STEPS steps.  Per step, as
# the reference's density() orders it: statistics, deposition (the Poisson
# solve every FINFET_POISSON_EVERY steps), surface rates, the carrier step;
# MultipleRefresh every 50 steps.  Phonon events tally heat throughout.
# Per window: the drain and source contact currents (the reference's
# `Current = ` of current_scatter_info, A), the section current through the
# middle third of the y planes (A), the electrons' mean y velocity (m/s) and
# mean energy (eV) from the statistic() sums, and the heat the carriers give
# the lattice (eV per step).
FINFET_WARMUP = 300
FINFET_WINDOWS = 8
FINFET_WINDOW_STEPS = 100
FINFET_POISSON_EVERY = 10
FINFET_MR_STEP = 50
FINFET_OBSERVABLES = ("drain_current_a", "source_current_a", "section_current_a", "drift_velocity_y_m_s",
                      "mean_energy_ev", "heat_ev_per_step")


def finfet_observables(window: dict, u: dict, dt: float, steps: int, ny: int) -> dict:
    """Window observables from its sums: contact tallies [contact][6]
    (NumParGen, CharGen, EnergyGen, NumParCatch, CharCatch, EnergyCatch),
    section currents lcurrent / rcurrent [ny + 1], the statistic() sums of
    the electrons (q, qvy, qe; summed over nodes) and the heat tallies
    (summed over nodes and carriers), all in the reference's normalised
    units.  The same function reads the engine's and the oracle's sums."""
    c = window["contact"]
    cur = lambda k: (c[k][1] - c[k][4]) / (dt * steps) * u["curr0"] * 1e-2
    lo, hi = ny // 3, 2 * ny // 3 + 1
    sec = (np.asarray(window["rcurrent"]) - np.asarray(window["lcurrent"]))[lo:hi].mean() / (dt * steps) * u["curr0"]
    q = window["electron_q"]
    return {"drain_current_a": cur(1), "source_current_a": cur(0), "section_current_a": float(sec),
            "drift_velocity_y_m_s": window["electron_qvy"] / q * u["spr0"] / u["time0"],
            "mean_energy_ev": window["electron_qe"] / q * u["eV0"],
            "heat_ev_per_step": window["heat"] * u["eV0"] / steps}


def run_finfet(precision: int, seed: int = 1, warmup: int = FINFET_WARMUP, windows: int = FINFET_WINDOWS,
               window_steps: int = FINFET_WINDOW_STEPS, device: int = 0) -> dict:
    """The FinFET protocol above on the GPU; returns the per-window
    observables and run totals."""
    import tempfile

    from . import Deck, Engine, decks

    with tempfile.TemporaryDirectory() as tmp:
        d = decks.finfet(tmp, total_step=warmup + windows * window_steps, heat_steps=0, compute_heat=False,
                         mr_step=FINFET_MR_STEP)
        deck = Deck(d["input"])
        root = Engine(max_particles=1, precision=precision, device=device)
        deck.prepare(root)
        carriers = int(deck.int_array("electron_num").sum() + deck.int_array("hole_num").sum())
        eng = Engine(max_particles=2 * carriers + 65536, precision=precision, device=device, like=root)
        deck.apply(eng)
        deck.seed(eng, seed)
        info = deck.info()
        eeff = deck.int_array("eeff_direction")
        refresh = (deck.int_array("refresh_electrons"), deck.int_array("refresh_holes"))
        deck.close()
    surf = dict(delta_m=0.4e-9, ail_m=1.5e-9, roughness=info["flag_surface_roughness"],
                phonon=info["flag_surface_phonon"])
    eng.set_refresh_targets(*refresh)
    eng._check(lib().mcb200_set_heat_tally(eng._ctx, 1), "mcb200_set_heat_tally")
    u = eng.units()
    dt = info["dt"]
    m = eng.mesh
    nodes = m.nnodes
    step = 0

    def advance(n):
        nonlocal step
        for _ in range(n):
            eng._check(lib().mcb200_stat_accumulate(eng._ctx), "mcb200_stat_accumulate")
            eng.deposit()
            if step % FINFET_POISSON_EVERY == 0:
                eng.solve_poisson_async(1e-10, 20000)
            eng.surface_rates(eeff, **surf)
            eng.step(step, seed, dt)
            if step % FINFET_MR_STEP == FINFET_MR_STEP - 1:
                eng.multiple_refresh(*refresh, step, seed, wait=False)
            step += 1

    eng.deposit()
    eng.solve_poisson(1e-10, 20000)
    eng._check(lib().mcb200_stat_begin(eng._ctx, max(warmup, 1)), "mcb200_stat_begin")
    advance(warmup)
    rows = []
    for _ in range(windows):
        eng.reset_tallies()
        eng._check(lib().mcb200_stat_begin(eng._ctx, window_steps), "mcb200_stat_begin")
        advance(window_steps)
        t = eng.tallies()
        w = {"contact": t["contact"][:info["n_contacts"]].tolist(), "lcurrent": t["lcurrent"].tolist(),
             "rcurrent": t["rcurrent"].tolist(), "electron_q": float(_stat(eng, "electron_q", nodes).sum()),
             "electron_qvy": float(_stat(eng, "electron_qvy", nodes).sum()),
             "electron_qe": float(_stat(eng, "electron_qe", nodes).sum()),
             "heat": float(t["heat_e"].sum() + t["heat_h"].sum())}
        rows.append(finfet_observables(w, u, dt, window_steps, m.ny))
    t = eng.tallies()
    out = {"precision": "fp32" if precision == FLIGHT_FP32 else "fp64", "windows": rows,
           "particles_end": eng.num_particles(), "no_tet": t["no_tet"], "zero_time": t["zero_time"],
           "caught": t["caught"]}
    eng.close()
    root.close()
    return out


def run_means(runs: list) -> list:
    """Each run's time average of every observable over its windows."""
    return [{key: float(np.mean([w[key] for w in r["windows"]])) for key in FINFET_OBSERVABLES} for r in runs]


def compare_runs(ref_runs: list, test_runs: list) -> dict:
    """Per observable, the test runs' mean time average against the
    reference runs' (compare_samples)."""
    a, b = run_means(ref_runs), run_means(test_runs)
    return {key: compare_samples([r[key] for r in a], [r[key] for r in b]) for key in FINFET_OBSERVABLES}


def finfet_report(seeds=(1, 2, 3, 4, 5, 6), device: int = 0, oracle_runs: list | None = None) -> dict:
    """FP32 flight against all-FP64 flight on the FinFET over independent
    seeds (and both against the reference's own runs when given)."""
    r64 = [run_finfet(FLIGHT_FP64, seed=s, device=device) for s in seeds]
    r32 = [run_finfet(FLIGHT_FP32, seed=s, device=device) for s in seeds]
    rep = {"fp64": r64, "fp32": r32, "fp32_vs_fp64": compare_runs(r64, r32)}
    if oracle_runs:
        rep["fp64_vs_oracle"] = compare_runs(oracle_runs, r64)
        rep["fp32_vs_oracle"] = compare_runs(oracle_runs, r32)
    return rep


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--electrons", type=int, default=100000)
    ap.add_argument("--warmup", type=int, default=300)
    ap.add_argument("--blocks", type=int, default=5)
    ap.add_argument("--block-steps", type=int, default=100)
    ap.add_argument("--seeds", type=int, default=8)
    ap.add_argument("--json", default=None)
    ap.add_argument("--finfet", action="store_true", help="the FinFET half instead of the bulk sweep")
    ap.add_argument("--finfet-seeds", type=int, default=6)
    ap.add_argument("--oracle-runs", default=None,
                    help="FinFET: a JSON file of the reference's runs of the same protocol ({'runs': [...]})")
    a = ap.parse_args()
    if a.finfet:
        oracle = None
        if a.oracle_runs:
            with open(a.oracle_runs) as f:
                oracle = json.load(f)["runs"]
        rep = finfet_report(seeds=tuple(range(1, a.finfet_seeds + 1)), oracle_runs=oracle)
        pairs = [k for k in ("fp32_vs_fp64", "fp64_vs_oracle", "fp32_vs_oracle") if k in rep]
        print(f"{'observable':>22} {'pair':>15} {'ref':>12} {'test':>12} {'rel':>9} {'sig':>6} {'limit':>6}")
        for key in FINFET_OBSERVABLES:
            for pair in pairs:
                e = rep[pair][key]
                print(f"{key:>22} {pair:>15} {e['ref']:12.5g} {e['test']:12.5g} {e['rel_error']:9.2e} "
                      f"{e['sigmas']:6.2f} {e['limit']:6.2f}")
        if a.json:
            with open(a.json, "w") as f:
                json.dump({k: rep[k] for k in pairs} | {"fp64_means": run_means(rep["fp64"]),
                                                        "fp32_means": run_means(rep["fp32"])}, f, indent=1)
        return
    rows = sweep(a.electrons, a.warmup, a.blocks, a.block_steps, seeds=a.seeds)
    print(f"{'E kV/cm':>8} {'vd FP64 m/s':>12} {'vd FP32':>12} {'rel':>8} {'sig':>5}  "
          f"{'E FP64 eV':>9} {'E FP32':>9} {'rel':>8} {'sig':>5}  {'imp rel':>8} {'ph rel':>8} {'valley sig':>10}")
    for r in rows:
        e = r["error"]
        v, en = e["drift_velocity_m_s"], e["mean_energy_ev"]
        print(f"{r['field_kv_cm']:8.0f} {v['ref']:12.4g} {v['test']:12.4g} {v['rel_error']:8.1e} {v['sigmas']:5.1f}  "
              f"{en['ref']:9.4f} {en['test']:9.4f} {en['rel_error']:8.1e} {en['sigmas']:5.1f}  "
              f"{e['impurity_per_particle_step']['rel_error']:8.1e} {e['phonon_per_particle_step']['rel_error']:8.1e} "
              f"{e['valley_max_sigmas']:10.1f}")
    if a.json:
        with open(a.json, "w") as f:
            json.dump(rows, f, indent=1)


if __name__ == "__main__":
    main()
