"""The bench's multi-process path on CPU: two ranks over gloo (the backend
bench.dist_init picks where there is no GPU), as torchrun would start them.
Replicas exchange nothing but the timing reductions: the whole-job
throughput is every rank's particle-steps over the slowest rank's time, and
the reference arm runs on rank 0 alone."""
import json
import os
import socket
import sys

import pytest
import torch.multiprocessing as tmp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench

    r, w, _ = bench.dist_init()
    res = {"rank": r, "world": w}
    res["sum"] = bench.dist_sum(float(r + 1), w)
    res["max"] = bench.dist_max(float(10 * r), w)
    bench.dist_barrier(w)
    # rank r flew 1e6 * (r + 1) particle-steps in 100 + 50 r ms of device time
    res["agg"] = bench.aggregate_throughput(1e6 * (r + 1), 100.0 + 50.0 * r, w)
    res["ref_arm_skipped"] = r != 0 and bench.reference_arm(None, r, w) is None
    bench._PG.destroy_process_group()
    with open(os.path.join(out_dir, f"rank{r}.json"), "w") as f:
        json.dump(res, f)


def test_two_gloo_ranks(tmp_path):
    world = 2
    tmp.start_processes(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn",
                        join=True)
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    for r in res:
        assert r["world"] == world
        assert r["sum"] == 3.0 and r["max"] == 10.0
        value, ms = r["agg"]
        assert ms == 150.0 and value == pytest.approx(3e6 / 0.150)
    assert res[1]["ref_arm_skipped"]
