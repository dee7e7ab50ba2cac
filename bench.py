#!/usr/bin/env python
"""Benchmark of the B200 carrier engine.

One JSON line on rank 0.  The headline workload is the self-consistent
n-FinFET (fin 10 nm x 30 nm, Lg 20 nm, 1 nm SiO2, S/D 1e20 cm^-3 with a
2 nm/dec roll-off into a 1e15 cm^-3 channel, nonuniform 80x50x40 mesh,
300k electrons + 50k holes requested -- 511k carriers after the reference's
per-cell minimum --, Vd 0.7 V, Vg 0.8 V, dt 0.2 fs, surface scattering on,
FP64 Poisson PCG every 10 steps, MultipleRefresh every 50).  A "step" is one
self-consistent step of mcb200_run_deck: statistics, deposition, Poisson (1
in 10), surface rates, carrier step (flight, GENERATE copies, removal, cell
sort), refresh.  Timed twice: FP32 flight and plain FP64 flight.

  value       FP32-flight particle-steps/s: particles flown over the timed
              steps / device time of those steps (CUDA events on the engine
              stream, an L2 eviction before every step, not timed: the
              working set is smaller than the 126 MB L2)
  fp64_plain  the same with FP64 flight; fp32_over_fp64 their ratio
  e2e         the same FP32 run through mcb200_run_deck with the contact
              tallies read back to the host after every step, host wall time
  roofline    flight kernel: 112 (FP32) / 160 (FP64) algorithmic bytes per
              particle-step (read + write of the state) / measured kernel
              time, against the measured HBM copy bandwidth
  bulk        the frozen-field bulk n-Si box (40x20x20 cells of 5 nm, 2M
              electrons, E_x = 10 kV/cm), flight-kernel throughput of both
              precisions
  cpu_baseline  the reference's own routines (CPU oracle: density_and_field
              every 10 steps + update_particle) on the same FinFET, one core

--impl reference times the same reference routines on all host cores, one
process per core.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "c-mc_electron_b200"))

METRIC = "particle-steps/s"
from mcb200.workloads import BULK_BOX as BOX  # noqa: E402

# read + write of the particle state: 80 B (FP64 plain), 56 B (FP32 flight)
BYTES_PER_PARTICLE_STEP = {"fp64": 160, "fp32": 112}
# DRAM bytes per particle-step of the flight kernel, from ncu captures of the
# same workload: the bulk box (its flight arm) and the FinFET (the headline)
PROFILE_TRAFFIC = {p: os.path.join(ROOT, "profiles", f"flight_{p}_bulk_traffic.json") for p in ("fp64", "fp32")}
FINFET_TRAFFIC = {p: os.path.join(ROOT, "profiles", f"flight_{p}_finfet_traffic.json") for p in ("fp64", "fp32")}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        finally:
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(rows)}


# ----------------------------------------------------------------- engine arm
def measure_precision(args, rank: int, world: int, device: int, precision: str):
    """Warm-up, timed steps and e2e steps of one flight precision on the bulk
    box; returns the measurements of this rank (maxima / sums over ranks)."""
    import mcb200
    from mcb200.workloads import bulk_box_engine

    seed = 1 + rank
    prec = mcb200.FLIGHT_FP32 if precision == "fp32" else mcb200.FLIGHT_FP64
    eng, dt, fields = bulk_box_engine(args.particles, seed, device, precision=prec)
    n0 = eng.num_particles()
    for s in range(args.warmup):
        eng.step(s, seed, dt)
    eng.sync()
    dist_barrier(world)
    eng.set_timing(True)
    eng.reset_tallies()
    with ClockSampler(device) as clocks:
        t0 = time.perf_counter()
        for s in range(args.warmup, args.warmup + args.steps):
            eng.step(s, seed, dt)
        eng.sync()
        wall = time.perf_counter() - t0
    tim = eng.timing()
    dist_barrier(world)
    step_ms = dist_max(tim["step_ms"], world)
    flight_ms_per_launch = tim["flight_ms"] / max(tim["flight_launches"], 1)
    tallies = eng.tallies()
    total_ps = dist_sum(tim["particles_flown"], world)
    # e2e: the public C ABI with host buffers; per step: pinned H2D of the
    # cell fields, one step, D2H of the tallies.
    try:
        import torch

        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    except Exception:  # torch without CUDA pinned memory: plain host buffers
        pin = lambda a: np.ascontiguousarray(a)
    e_h, h_h, rho_h = (pin(a) for a in fields)
    h2d = e_h.nbytes + h_h.nbytes + rho_h.nbytes
    e2e_steps = max(3, min(args.steps, 20))
    base = args.warmup + args.steps
    dist_barrier(world)
    t0 = time.perf_counter()
    d2h = 0
    for s in range(base, base + e2e_steps):
        eng.set_fields(e_h, h_h, rho_h)
        eng.step(s, seed, dt)
        eng.tallies()
        d2h = 8 * (16 + 16 * 6 + 2 * (eng.mesh.ny + 1) + 2 * eng.mesh.nnodes)
    e2e_wall = dist_max(time.perf_counter() - t0, world)
    e2e_ps = dist_sum(float(eng.num_particles()) * e2e_steps, world)
    bytes_ps = BYTES_PER_PARTICLE_STEP[precision]
    per_launch = tim["particles_flown"] / max(tim["flight_launches"], 1)
    achieved = bytes_ps * per_launch / (flight_ms_per_launch * 1e-3) / 1e9
    traffic = None
    try:
        with open(PROFILE_TRAFFIC[precision]) as f:
            traffic = json.load(f)["dram_bytes_per_particle_step"] * per_launch
    except Exception:
        pass
    out = dict(n0=n0, value=total_ps / (step_ms * 1e-3), step_ms=step_ms, wall=wall,
               flight_ms_per_launch=flight_ms_per_launch, launches=int(tim["launches"]),
               clocks=clocks.summary(), e2e=e2e_ps / e2e_wall, h2d=h2d, d2h=d2h, achieved=achieved,
               traffic=traffic, bytes=bytes_ps,
               events=tallies["events"] / max(tim["particles_flown"], 1), caught=tallies["caught"],
               zero_time=tallies["zero_time"])
    eng.close()
    return out


FINFET_POISSON_EVERY = 10
FINFET_CARRIERS = 511200  # 300k e- + 50k h+ requested, raised by the per-cell minimum (compute_par_num)


def finfet_config(world: int) -> dict:
    """The FinFET workload both arms run (engine and reference)."""
    return {"workload": "n-FinFET self-consistent: fin 10x30 nm, Lg 20 nm, 1 nm SiO2, S/D 1e20 cm^-3 (2 nm/dec), "
                        "channel 1e15 cm^-3, 80x50x40 nonuniform mesh (0.5 nm channel, 2 nm contacts), 300k e- + "
                        "50k h+ requested (511,200 carriers with the per-cell minimum), Vd 0.7 V, Vg 0.8 V, dt 0.2 "
                        "fs, surface scattering, Poisson every 10 steps, MultipleRefresh every 50",
            "carriers": FINFET_CARRIERS,
            "l2": "L2 evicted (256 MB write) before every timed step on the GPU, eviction not timed",
            "parallelism": f"replicas{world}"}
PHASE_PROFILE_STEPS = 60  # steps of the phase-split run (each phase waited for)
FLUSH_BYTES = 256 << 20  # > 126 MB L2


def finfet_run(args, device: int, precision: str, readback: bool = False, profile_steps: int = 0) -> dict:
    """One run of the FinFET deck.  profile_steps > 0: a short run that waits
    for the GPU after every phase, for the per-phase device time split only."""
    import mcb200
    from mcb200 import decks

    steps = profile_steps if profile_steps else args.steps
    with tempfile.TemporaryDirectory() as tmp:
        d = decks.finfet(tmp, total_step=args.warmup + steps + 1, heat_steps=0, stat_step=100000)
        prec = mcb200.FLIGHT_FP32 if precision == "fp32" else mcb200.FLIGHT_FP64
        with ClockSampler(device) as clocks:
            rep = mcb200.run_deck(d["input"], device=device, precision=prec, max_steps=args.warmup + steps,
                                  warmup_steps=args.warmup, max_heat_steps=0, poisson_every=FINFET_POISSON_EVERY,
                                  write_outputs=False, readback_every_step=readback,
                                  flush_l2_bytes=0 if (readback or profile_steps) else FLUSH_BYTES,
                                  profile_phases=bool(profile_steps))
        rep["clocks"] = clocks.summary()
    return rep


def engine_arm(args, rank: int, world: int, device: int):
    runs = {p: finfet_run(args, device, p) for p in ("fp64", "fp32")}
    e2e = finfet_run(args, device, "fp32", readback=True) if args.workload == "all" else runs["fp32"]
    phases = finfet_run(args, device, "fp32", profile_steps=PHASE_PROFILE_STEPS)
    peak, peak_kind = measured_peaks()
    value = {}
    for p, r in runs.items():
        value[p], _ = aggregate_throughput(r["timed_particle_steps"], r["timed_device_ms"], world)

    def roof(r, p):
        # the flight's device time is sampled on one timed step in ten (events
        # on every step would cost the others their overlapped launches); one
        # main flight per step
        per_launch = r["timed_particle_steps"] / max(r["timed_steps"], 1)
        kernel_ms = r["timed_flight_ms"] / max(r["timed_flight_launches"], 1)
        achieved = BYTES_PER_PARTICLE_STEP[p] * per_launch / (kernel_ms * 1e-3) / 1e9
        traffic = None
        try:
            with open(FINFET_TRAFFIC[p]) as f:
                traffic = json.load(f)["dram_bytes_per_particle_step"] * per_launch
        except Exception:
            pass
        return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "kernel": f"flight_kernel<{'float' if p == 'fp32' else 'double'}>",
                "peak_kind": peak_kind, "bytes_per_unit": BYTES_PER_PARTICLE_STEP[p],
                "kernel_ms_per_launch": kernel_ms, "particles_per_launch": per_launch}

    r32, r64 = runs["fp32"], runs["fp64"]
    nodes = 81 * 51 * 41
    cg = {"solves": r32["poisson_solves"], "iterations": r32["poisson_iterations"],
          "max_rel_residual": r32["poisson_max_residual"]}
    bulk = {}
    for p in (("fp64", "fp32") if args.workload == "all" else ()):
        m = measure_precision(args, rank, world, device, p)
        bulk[p] = {"value": m["value"], "flight_ms_per_launch": m["flight_ms_per_launch"],
                   "roofline_frac": m["achieved"] / peak, "achieved_gbs": m["achieved"],
                   "particles": m["n0"], "events_per_particle_step": m["events"]}
    e2e_ps = dist_sum(e2e["timed_particle_steps"], world) / dist_max(e2e["timed_wall_s"], world)
    return {
        "metric": METRIC, "value": value["fp32"], "unit": "particle-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r32["timed_device_ms"] / max(r32["timed_steps"], 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": finfet_config(world),
        "precision": "fp32-flight (FP64 energy / time bookkeeping); fp64_plain: all-FP64 flight",
        "carriers_initial": r32["initial_particles"],
        "e2e": {"value": e2e_ps, "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 16 * 6 * 8,
                "note": "mcb200_run_deck (the main input.txt path) with the contact tallies read back every step "
                        "(pipelined: a step's 768 B are read while the next step runs); "
                        "the deck is read and uploaded once, the self-consistent state stays on the device, so no "
                        "per-step host input exists"},
        "roofline": roof(r32, "fp32"),
        "gpu_launches": int(r32["timed_launches"]),
        "clocks": r32["clocks"],
        "fp64_plain": {"value": value["fp64"], "ms_per_step": r64["timed_device_ms"] / max(r64["timed_steps"], 1),
                       "dtype": "f64", "roofline": roof(r64, "fp64"), "gpu_launches": int(r64["timed_launches"]),
                       "clocks": r64["clocks"]},
        "fp32_over_fp64": value["fp32"] / value["fp64"],
        "poisson": cg,
        "phase_s_fp32": phases["phase_s"], "phase_profile_steps": PHASE_PROFILE_STEPS + args.warmup,
        "bulk": bulk,
        "bulk_fp32_over_fp64": bulk["fp32"]["value"] / bulk["fp64"]["value"] if bulk else None,
    }


# ------------------------------------------------------------ batching
BATCH_MEMBERS = 64
BATCH_STEPS = 40


def batch_arm(args, device: int) -> dict:
    """Many simulations at once: 64 seeded members, half frozen-field bulk
    boxes (20^3 to 80x40x50 cells, E_x 1-100 kV/cm), half self-consistent
    FinFETs (Lg 15/20/30 nm, Vg 0-0.8 V), particle counts log-uniform in
    5k-500k, FP32 flight.  Full timesteps through the batch (one flight
    launch per step for all members, steps replayed from CUDA graphs, launch
    shapes, overlap and solve pairing from the autotuner) against the same
    members stepped one by one on their own streams, the two timed in
    interleaved windows of 20 steps (batched, alone, alone, batched).  Device
    time between batch marks (every member's stream joined), particle-steps
    from the members' device counters."""
    import mcb200
    from mcb200 import batching

    t0 = time.perf_counter()
    members, root = batching.build_mix(n=BATCH_MEMBERS, seed=4, precision=mcb200.FLIGHT_FP32)
    setup_s = time.perf_counter() - t0
    batch = mcb200.Batch([(m.eng, m.cfg) for m in members])
    batch.use_graphs(True)
    s0 = batch.info()["steps"]
    tune = batch.autotune(10)
    for m in members:
        m.step += batch.info()["steps"] - s0

    def window(run, k):
        ps0 = batching.particle_steps(members)
        batch.mark(0)
        run(k)
        batch.mark(1)
        return batching.particle_steps(members) - ps0, batch.elapsed_ms(0, 1)

    run_b = lambda k: batching.run_batched(batch, members, k)  # noqa: E731
    run_a = lambda k: batching.run_alone(members, k)  # noqa: E731
    run_b(10)  # warm-ups: graphs of every step kind, first launches
    run_a(10)
    # The members' particle counts drift as they evolve, so the two arms are
    # timed in interleaved windows (batched, alone, alone, batched, ...): a
    # steady drift weighs on both alike.
    tot = {"b": [0, 0.0], "a": [0, 0.0]}
    order = ["b", "a", "a", "b"]
    windows = []
    with ClockSampler(device) as clocks:
        for arm in order:
            ps, ms = window(run_b if arm == "b" else run_a, BATCH_STEPS // 2)
            tot[arm][0] += ps
            tot[arm][1] += ms
            windows.append({"arm": "batched" if arm == "b" else "alone", "ms_per_step": ms / (BATCH_STEPS // 2),
                            "particles_per_step": ps / (BATCH_STEPS // 2)})
    batched, ms_b = tot["b"][0] / (tot["b"][1] * 1e-3), tot["b"][1] / BATCH_STEPS
    alone, ms_a = tot["a"][0] / (tot["a"][1] * 1e-3), tot["a"][1] / BATCH_STEPS
    info = batch.info()
    kinds = [m.kind for m in members]
    out = {"metric": "particle-steps/s", "members": len(members), "bulk": kinds.count("bulk"),
           "finfet": kinds.count("finfet"), "particles": int(sum(m.desc["particles"] for m in members)),
           "value": batched, "ms_per_step": ms_b, "unbatched_value": alone, "unbatched_ms_per_step": ms_a,
           "batched_over_unbatched": batched / alone, "steps": BATCH_STEPS, "windows": windows, "autotune": tune,
           "graph_captures": info["graph_captures"], "graph_replays": info["graph_replays"],
           "setup_s": setup_s, "clocks": clocks.summary(), "dtype": "f32", "data": "synthetic",
           "config": "64 members (seed 4): bulk n-Si boxes 20^3-80x40x50 cells, E_x U[1,100] kV/cm, and "
                     "self-consistent n-FinFETs Lg {15,20,30} nm, Vg U[0,0.8] V, Vd 0.7 V, surface scattering, "
                     "Poisson every 10 steps (staggered), MultipleRefresh every 50; N log-uniform 5k-500k "
                     "(FinFETs at least one electron per silicon cell); working set > L2"}
    batch.close()
    for m in members:
        m.eng.close()
    root.close()
    return out


# ------------------------------------------------------------ serving
SERVE_REQUESTS = 32
SERVE_MAX_STEPS = 2000
SERVE_QUANTUM = 50


def serve_arm(args, device: int) -> dict:
    """A 32-point bias sweep served by continuous batching: n-FinFET requests
    (Vg 0-0.8 V in 0.05 V steps x Vd {0.05, 0.7} V x Lg {15, 20, 30} nm,
    50k-1M particles log-uniform) arriving as a Poisson process of 4 req/s
    (seed 5); FP32 flight, HBM budget 160 GB, one Ids window per 50-step
    round (net flux through the middle third of the section planes), each
    request done when stderr(Ids) < 1% of |Ids| after 6 transient windows
    (2 after a warm start) or at the step cap (2000 by default); a request
    warm-starts from the nearest converged bias of its Lg, failing that from
    the nearest running request of its Lg past its transient.  Latency = completion - arrival
    (server clock); throughput = particle-steps over the rounds' device time."""
    import mcb200
    from mcb200 import serving

    with tempfile.TemporaryDirectory() as tmp:
        reqs = serving.make_requests(tmp, n=SERVE_REQUESTS, seed=5, rate=4.0)
        srv = mcb200.Server(device=device, precision=mcb200.FLIGHT_FP32, quantum_steps=SERVE_QUANTUM)
        with ClockSampler(device) as clocks:
            res, st, wall = serving.serve(srv, reqs, max_wall_s=900, max_steps=args.serve_max_steps, min_windows=5,
                                          warm_windows_cold=6, warm_windows_warm=2, poisson_every=10,
                                          target_rel_err=0.01, ids_estimator=mcb200.IDS_SECTIONS,
                                          warm_start=mcb200.WARM_SETTLED)
        srv.close()
    lat = serving.latency_summary(res)
    status = [r["status"] for r in res]
    by_id = {r["id"]: r for r in reqs}
    rel = [abs(r["ids_stderr"] / r["ids"]) if r["ids"] else float("inf") for r in res]
    per_request = [[by_id[r["id"]]["lg_nm"], by_id[r["id"]]["vg"], by_id[r["id"]]["vd"], r["particles"], r["steps"],
                    round(e, 4), r["status"], round(r["done_s"] - r["arrival_s"], 2)] for r, e in zip(res, rel)]
    return {"metric": "bias-point latency", "unit": "s", "p50_s": lat.get("p50_s"), "p99_s": lat.get("p99_s"),
            "mean_s": lat.get("mean_s"), "requests": SERVE_REQUESTS, "completed": len(res),
            "converged": status.count(mcb200.SERVE_CONVERGED), "step_limited": status.count(mcb200.SERVE_STEP_LIMIT),
            "warm_started": sum(1 for r in res if r["warm_from"]),
            "throughput_particle_steps_per_s": st["particle_steps"] / (st["device_ms"] * 1e-3),
            "particle_steps": st["particle_steps"], "rounds": st["rounds"], "wall_s": wall,
            "median_rel_stderr": float(statistics.median(rel)) if res else None,
            "per_request": per_request,
            "per_request_fields": ["lg_nm", "vg", "vd", "particles", "steps", "rel_stderr", "status", "latency_s"],
            "clocks": clocks.summary(),
            "config": "32 FinFET bias points, Poisson arrivals 4 req/s, 50k-1M particles, 160 GB budget, "
                      f"target 1% Ids stderr, {args.serve_max_steps}-step cap, 50-step rounds, FP32 flight, "
                      "warm starts from converged or settled requests of the same Lg"}


# ------------------------------------------------------------ reference (CPU)
def _oracle_sample(args):
    """One CPU process: the reference's routines on the FinFET deck of the
    engine arm (density_and_field every FINFET_POISSON_EVERY steps --
    BiCGSTAB standing in for KLU -- and update_particle every step); returns
    (particle-steps, seconds).  The deck's initialisation is not timed."""
    seed, electrons, holes, steps = args
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from mcb200 import decks
    from oracle_bridge import Oracle

    with tempfile.TemporaryDirectory() as tmp:
        deck = decks.finfet(tmp, electrons=electrons, holes=holes)
        orc = Oracle()
        orc.init(deck["input"], seed=seed)
    n = len(orc.particles()["x"])
    t0 = time.perf_counter()
    ps = 0
    for s in range(steps):
        if s % FINFET_POISSON_EVERY == 0:
            orc.density_and_field()
        orc.flight_step(s)
        ps += n
        n = len(orc.particles()["x"]) if s % FINFET_POISSON_EVERY == FINFET_POISSON_EVERY - 1 else n
    return ps, time.perf_counter() - t0


FINFET_REQUEST = (300000, 50000)  # electrons, holes requested in the deck


def cpu_baseline(steps: int = 10):
    """The reference's routines on the engine arm's FinFET (511,200 carriers),
    one core: one Poisson solve and `steps` flights (about 10-15 s)."""
    ps, t = _oracle_sample((99, *FINFET_REQUEST, steps))
    return {"value": ps / t, "unit": "particle-steps/s", "cores": 1, "kind": "reference",
            "sample": f"the reference's density_and_field (every {FINFET_POISSON_EVERY} steps) + update_particle on "
                      f"the engine arm's FinFET deck ({FINFET_CARRIERS} carriers), {steps} steps, {t:.1f} s, "
                      "one core"}


def reference_arm(args, rank: int, world: int):
    if rank != 0:
        return None
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    steps = max(3, min(args.steps, 20))
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        res = pool.map(_oracle_sample, [(1000 + i, *FINFET_REQUEST, steps) for i in range(cores)])
    total_ps = sum(r[0] for r in res)
    wall = max(r[1] for r in res)
    value = total_ps / wall
    return {
        "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": steps,
        "warmup": args.warmup, "ms_per_step": wall / steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": finfet_config(world),
        "precision": "all-FP64 (the reference's CPU code)",
        "processes": cores,
        "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": cores, "kind": "reference",
                         "sample": f"{cores} independent processes, each {steps} steps of the reference's "
                                   f"density_and_field (every {FINFET_POISSON_EVERY} steps) + update_particle on the "
                                   f"engine arm's FinFET deck ({FINFET_CARRIERS} carriers)"},
        "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ------------------------------------------------------------ distribution
_PG = None


_ON_GPU = False


def dist_init():
    """One process per GPU (torchrun's RANK / WORLD_SIZE / LOCAL_RANK):
    NCCL between GPUs, gloo where there is no GPU (the CPU tests)."""
    global _PG, _ON_GPU
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        _ON_GPU = torch.cuda.is_available()
        if _ON_GPU:
            torch.cuda.set_device(local)
        dist.init_process_group("nccl" if _ON_GPU else "gloo", timeout=datetime.timedelta(seconds=300))
        _PG = dist
    return rank, world, local


def aggregate_throughput(particle_steps: float, device_ms: float, world: int):
    """Whole-job throughput of the replicas: every rank's particle-steps over
    the slowest rank's device time.  Returns (particle-steps/s, max ms)."""
    total = dist_sum(float(particle_steps), world)
    ms = dist_max(float(device_ms), world)
    return total / (ms * 1e-3), ms


def dist_barrier(world):
    if world > 1 and _PG is not None:
        _PG.barrier()


def _reduce(v: float, world: int, op):
    if world == 1 or _PG is None:
        return v
    import torch

    t = torch.tensor([v], dtype=torch.float64, device="cuda" if _ON_GPU else "cpu")
    _PG.all_reduce(t, op=op)
    return float(t.item())


def dist_max(v, world):
    return _reduce(v, world, _PG.ReduceOp.MAX if _PG else None)


def dist_sum(v, world):
    return _reduce(v, world, _PG.ReduceOp.SUM if _PG else None)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--particles", type=int, default=2_000_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="all", choices=["all", "finfet", "finfet32", "batch", "serve"],
                    help="finfet: only the two FinFET arms (no e2e rerun, no bulk box): for profiling; "
                         "finfet32: one FP32 run of the FinFET deck alone (profiling); batch: only the batching arm")
    ap.add_argument("--serve-max-steps", type=int, default=SERVE_MAX_STEPS,
                    help="serving: a request's step cap (it completes earlier when stderr(Ids) < 1%% of Ids)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    rank, world, local = dist_init()
    if args.impl == "reference":
        out = reference_arm(args, rank, world)
    elif args.workload == "batch":
        out = batch_arm(args, local)
    elif args.workload == "serve":
        out = serve_arm(args, local)
    elif args.workload == "finfet32":
        r = finfet_run(args, local, "fp32")
        out = {"workload": "finfet32", "ms_per_step": r["timed_device_ms"] / max(r["timed_steps"], 1),
               "timed_particle_steps": r["timed_particle_steps"], "timed_steps": r["timed_steps"],
               "flight_ms_per_launch": r["timed_flight_ms"] / max(r["timed_flight_launches"], 1),
               "clocks": r["clocks"]}
    else:
        out = engine_arm(args, rank, world, local)
        if args.workload == "all":
            out["batch"] = batch_arm(args, local)
            out["serving"] = serve_arm(args, local)
            out["p50_latency_s"] = out["serving"]["p50_s"]
            out["p99_latency_s"] = out["serving"]["p99_s"]
        if rank == 0 and not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_baseline()
    if rank == 0 and out is not None:
        print(json.dumps(out), flush=True)
    if _PG is not None:
        _PG.destroy_process_group()


if __name__ == "__main__":
    main()
