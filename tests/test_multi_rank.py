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
