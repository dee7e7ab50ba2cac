"""Serving bias-point requests (mcb200_server_*): an open-loop client.

make_requests(): a seeded stream of n-FinFET bias-point requests -- Vg in
{0, 0.05, ..., 0.8} V x Vd in {0.05, 0.7} V x gate length in {15, 20, 30}
nm, particle counts log-uniform between two bounds (a FinFET holds at least
one electron per silicon cell) -- arriving as a Poisson process of a given
rate.  Requests of one gate length form a family (one mesh), so a request
can warm-start from the converged ensemble of the nearest bias of its
family.

serve(): the open-loop client.  Between rounds it submits every request
whose arrival time has passed (its arrival time, not the submission time,
is what latency counts from), sleeps while the server is idle and the next
arrival is in the future, and collects the results.
"""
from __future__ import annotations

import math
import os
import time

import numpy as np

from . import Server
from . import decks

VG = [round(0.05 * i, 2) for i in range(17)]
VD = [0.05, 0.7]
LG = [15.0, 20.0, 30.0]


def make_requests(tmp: str, n=32, seed=5, rate=4.0, n_min=50_000, n_max=1_000_000, mr_step=50):
    """n requests (distinct bias points) with Poisson arrivals; each writes
    its deck under tmp.  Returns [dict(input, family, bias, seed, arrival,
    lg_nm, vg, vd, particles)]."""
    rng = np.random.default_rng(seed)
    grid = [(lg, vg, vd) for lg in LG for vg in VG for vd in VD]
    pick = rng.choice(len(grid), size=n, replace=False)
    gaps = rng.exponential(1.0 / rate, size=n)
    arrivals = np.cumsum(gaps) - gaps[0]
    counts = np.exp(rng.uniform(math.log(n_min), math.log(n_max), n)).astype(int)
    out = []
    for i in range(n):
        lg, vg, vd = grid[pick[i]]
        d = decks.finfet(os.path.join(tmp, f"req{i}"), electrons=int(counts[i]), holes=max(int(counts[i]) // 6, 1),
                         vg=vg, vd=vd, lg_nm=lg, min_per_cell=(1, 0), compute_heat=False, mr_step=mr_step)
        out.append(dict(input=d["input"], family=f"lg{lg:g}", bias=(vg, vd), seed=5000 + i,
                        arrival=float(arrivals[i]), lg_nm=lg, vg=vg, vd=vd, particles=int(counts[i])))
    return out


def serve(server: Server, requests, max_wall_s: float = 600.0, **submit_kw):
    """Run the server on the request stream until every request finished
    (or max_wall_s passed).  Returns (results, stats, wall_s)."""
    order = sorted(requests, key=lambda r: r["arrival"])
    t0 = server.now()
    nxt, results = 0, []
    while len(results) < len(order):
        now = server.now() - t0
        if now > max_wall_s:
            break
        while nxt < len(order) and order[nxt]["arrival"] <= now:
            r = order[nxt]
            r["id"] = server.submit(r["input"], r["family"], r["bias"], r["seed"], arrival_s=t0 + r["arrival"],
                                    **submit_kw)
            nxt += 1
        active, pending = server.round()
        results += server.results()
        if active == 0 and pending == 0 and nxt < len(order):
            time.sleep(max(0.0, order[nxt]["arrival"] - (server.now() - t0)))
    return results, server.stats(), server.now() - t0


def latency_summary(results) -> dict:
    lat = np.array([r["done_s"] - r["arrival_s"] for r in results if r["status"] > 0])
    if lat.size == 0:
        return {}
    return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "max_s": float(lat.max()), "completed": int(lat.size)}
