"""Host logic of `bench.py --gpus N` (one replica per rank), on CPU with the
gloo backend and two ranks: the device times are reduced to their maximum
over the ranks, and the whole-job rate counts every rank's cells over that
slowest time. The reference arm runs on rank 0 only.
"""
from __future__ import annotations

import io
import json
import os
import socket
import sys
from contextlib import redirect_stdout
from pathlib import Path

import pytest
import torch.multiprocessing as mp

REPO = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str) -> None:
    import datetime
    import torch.distributed as D
    sys.path.insert(0, str(REPO))
    import bench
    D.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                         timeout=datetime.timedelta(seconds=60))
    bench._DIST["on"] = True
    local_ms = [12.5, 20.0][rank]                    # rank 1 is the slow replica
    rate, max_ms = bench.whole_job_rate(local_ms, world, cells=1000, steps=10)
    bench.dist_barrier()
    Path(out_dir, f"rank{rank}.json").write_text(json.dumps({"rate": rate, "max_ms": max_ms}))
    D.barrier()
    D.destroy_process_group()


def test_two_ranks_take_the_slowest_time(tmp_path):
    world, port = 2, _free_port()
    mp.start_processes(_rank_main, args=(world, port, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    res = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(world)]
    for r in res:
        assert r["max_ms"] == 20.0
        assert r["rate"] == pytest.approx(world * 1000 * 10 / 20e-3)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, str(REPO))
    import bench
    assert not bench.dist_on()
    rate, max_ms = bench.whole_job_rate(5.0, 1, cells=100, steps=4)
    assert max_ms == 5.0 and rate == pytest.approx(100 * 4 / 5e-3)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    sys.path.insert(0, str(REPO))
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0"])
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.main()                                  # returns at once: no work, no line
    assert buf.getvalue() == ""


def test_ensemble_shards_cover_every_case_once_and_balance_cost():
    sys.path.insert(0, str(REPO / "2d-vector-vorticity-model_b200"))
    from vvm_b200.ensemble import ensemble_specs, shard_by_cost
    specs = ensemble_specs(256, 3)
    assert len(specs) == 256 and specs == ensemble_specs(256, 3)
    assert {s["NX"] for s in specs} <= {256, 512, 1024, 2048} and {s["NZ"] for s in specs} <= {64, 96, 128}
    assert all(1.0 <= s["amp"] <= 3.0 and 0.2 <= s["xc_frac"] <= 0.8 and 1000 <= s["radius"] <= 3000
               for s in specs)
    costs = [s["NX"] * s["NZ"] for s in specs]
    for world in (1, 2, 4, 8):
        shards = shard_by_cost(costs, world)
        flat = sorted(i for sh in shards for i in sh)
        assert flat == list(range(256))
        loads = [sum(costs[i] for i in sh) for sh in shards]
        assert max(loads) - min(loads) <= max(costs)   # greedy longest-first bound


def _shard_rank(rank, world, port, out_dir):
    import datetime
    import torch.distributed as D
    sys.path.insert(0, str(REPO / "2d-vector-vorticity-model_b200"))
    from vvm_b200.ensemble import ensemble_specs, shard_by_cost
    D.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                         timeout=datetime.timedelta(seconds=60))
    specs = ensemble_specs(64, 7)
    mine = shard_by_cost([s["NX"] * s["NZ"] for s in specs], world)[rank]
    Path(out_dir, f"shard{rank}.json").write_text(json.dumps(mine))
    D.barrier()
    D.destroy_process_group()


def test_ranks_compute_disjoint_shards_without_exchange(tmp_path):
    world, port = 2, _free_port()
    mp.start_processes(_shard_rank, args=(world, port, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    a = json.loads((tmp_path / "shard0.json").read_text())
    b = json.loads((tmp_path / "shard1.json").read_text())
    assert not set(a) & set(b) and sorted(a + b) == list(range(64))
