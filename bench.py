#!/usr/bin/env python
"""Benchmark of the B200 carrier engine on its frozen-field bulk workload.

One JSON line on rank 0.  A "step" is one transport step (mcb200_step:
flight of every particle over dt, mid-step copies, removal, counting sort by
cell) of the bulk n-Si box: 40x20x20 cells of 5 nm, N_D = 1e17 cm^-3, 300 K,
frozen uniform E_x = 10 kV/cm, dt = 1 fs, REFLECT on every face (the
reference's bulk physics), with the electron ensemble scaled so the
particle store exceeds the 126 MB L2.  The same workload is timed twice:
plain FP64 flight (80 B / particle, the reference's arithmetic) and FP32
flight (56 B / particle, float kinematics and rate lookups, FP64 energy and
time bookkeeping).

  value       FP32-flight particle-steps/s of the whole job, state resident
              in HBM, device time of the timed steps (CUDA events on the
              engine stream); fp64_plain.value is the FP64 arm, and
              fp32_over_fp64 their ratio
  e2e         the same metric through the C ABI with host buffers: each
              step uploads the step's cell fields from pinned memory and
              reads the tallies back
  roofline    flight kernel: 112 (FP32) / 160 (FP64) algorithmic bytes per
              particle-step (read + write of the state) / measured kernel
              time, against the measured HBM copy bandwidth
  cpu_baseline  the reference's own update_particle() (CPU oracle, one core)
              on a bounded sample of the same box

--impl reference times the reference's CPU implementation (the oracle built
from its sources) on all host cores, one process per core.
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
PROFILE_TRAFFIC = {p: os.path.join(ROOT, "profiles", f"flight_{p}_bulk_traffic.json") for p in ("fp64", "fp32")}


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


def engine_arm(args, rank: int, world: int, device: int):
    fp64 = measure_precision(args, rank, world, device, "fp64")
    fp32 = measure_precision(args, rank, world, device, "fp32")
    peak, peak_kind = measured_peaks()
    box = f"bulk n-Si box {BOX['nx']}x{BOX['ny']}x{BOX['nz']} cells of 5 nm, N_D=1e17 cm^-3, E_x=10 kV/cm frozen, " \
          f"300 K, dt=1 fs, {fp32['n0']} electrons per GPU"
    roof = lambda m: {"bound": "hbm", "achieved": m["achieved"], "peak": peak, "unit": "GB/s",
                      "frac": m["achieved"] / peak, "traffic": m["traffic"], "kernel": "flight_kernel",
                      "peak_kind": peak_kind, "bytes_per_unit": m["bytes"]}
    return {
        "metric": METRIC, "value": fp32["value"], "unit": "particle-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": fp32["step_ms"] / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": box + "; FP32 flight (FP64 energy/time bookkeeping) vs plain FP64 flight",
                   "particles_per_gpu": fp32["n0"], "precision": "fp32-flight",
                   "l2": "particle store larger than L2 (56 B / 80 B x particles)",
                   "parallelism": f"replicas{world}"},
        "e2e": {"value": fp32["e2e"], "unit": "particle-steps/s", "h2d_bytes_per_step": fp32["h2d"],
                "d2h_bytes_per_step": fp32["d2h"]},
        "roofline": roof(fp32),
        "gpu_launches": fp32["launches"],
        "clocks": fp32["clocks"],
        "fp64_plain": {"value": fp64["value"], "ms_per_step": fp64["step_ms"] / args.steps, "dtype": "f64",
                       "e2e": fp64["e2e"], "roofline": roof(fp64), "gpu_launches": fp64["launches"],
                       "clocks": fp64["clocks"], "events_per_particle_step": fp64["events"]},
        "fp32_over_fp64": fp32["value"] / fp64["value"],
        "flight_ms_per_launch": fp32["flight_ms_per_launch"],
        "events_per_particle_step": fp32["events"],
        "fp32_zero_time_catches": fp32["zero_time"],
        "wall_s": fp32["wall"] + fp64["wall"],
    }


# ------------------------------------------------------------ reference (CPU)
def _oracle_sample(args):
    """One CPU process: the reference's update_particle on the bulk box
    (electrons only), `steps` steps; returns (particle-steps, seconds)."""
    seed, electrons, steps, warmup = args
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from mcb200 import decks
    from oracle_bridge import Oracle

    with tempfile.TemporaryDirectory() as tmp:
        deck = decks.bulk_box(tmp, nx=BOX["nx"], ny=BOX["ny"], nz=BOX["nz"], electrons=electrons, holes=0)
        orc = Oracle()
        orc.init(deck["input"], seed=seed)
    p = orc.particles()
    keep = p["type"] == 0
    orc.set_particles({k: v[keep] for k, v in p.items()}, orc.scalar("dt"))
    f0 = orc.scalar("field0")
    n = len(orc.array("c_field_x"))
    orc.set_array("c_field_x", np.full(n, BOX["field_v_per_m"] / f0))
    if warmup:
        orc.time_update_particle(warmup)
    t = orc.time_update_particle(steps)
    return int(keep.sum()) * steps, t


def cpu_baseline(target_s: float = 12.0):
    electrons = 20000
    ps, t = _oracle_sample((99, electrons, 2, 0))
    steps = max(3, int(target_s / max(t / 2, 1e-6)))
    ps, t = _oracle_sample((99, electrons, min(steps, 2000), 0))
    return {"value": ps / t, "unit": "particle-steps/s", "cores": 1, "kind": "reference",
            "sample": f"reference update_particle()+compute_cell_charge() on the same box, {electrons} "
                      f"electrons, {min(steps, 2000)} steps, {t:.1f} s on one core"}


def reference_arm(args, rank: int, world: int):
    if rank != 0:
        return None
    cores = os.cpu_count() or 1
    per_step_particles = 20000
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        res = pool.map(_oracle_sample, [(1000 + i, per_step_particles, args.steps, args.warmup) for i in range(cores)])
    total_ps = sum(r[0] for r in res)
    wall = max(r[1] for r in res)
    value = total_ps / wall
    return {
        "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": wall / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": {"workload": f"bulk n-Si box {BOX['nx']}x{BOX['ny']}x{BOX['nz']} cells of 5 nm, N_D=1e17 cm^-3, "
                               "E_x=10 kV/cm frozen, 300 K, dt=1 fs, FP64 (reference CPU code)",
                   "particles_per_process": per_step_particles, "processes": cores},
        "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": cores, "kind": "reference",
                         "sample": f"{cores} independent processes x {per_step_particles} electrons x "
                                   f"{args.steps} steps of the reference's update_particle()"},
        "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ------------------------------------------------------------ distribution
_PG = None


def dist_init():
    global _PG
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        _PG = dist
    return rank, world, local


def dist_barrier(world):
    if world > 1 and _PG is not None:
        _PG.barrier()


def _reduce(v: float, world: int, op):
    if world == 1 or _PG is None:
        return v
    import torch

    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    _PG.all_reduce(t, op=op)
    return float(t.item())


def dist_max(v, world):
    return _reduce(v, world, _PG.ReduceOp.MAX if _PG else None)


def dist_sum(v, world):
    return _reduce(v, world, _PG.ReduceOp.SUM if _PG else None)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--particles", type=int, default=2_000_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    rank, world, local = dist_init()
    if args.impl == "reference":
        out = reference_arm(args, rank, world)
    else:
        out = engine_arm(args, rank, world, local)
        if rank == 0 and not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_baseline()
    if rank == 0 and out is not None:
        print(json.dumps(out), flush=True)
    if _PG is not None:
        _PG.destroy_process_group()


if __name__ == "__main__":
    main()
