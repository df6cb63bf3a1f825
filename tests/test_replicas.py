"""The multi-GPU replica path's host logic, with two gloo ranks on CPU.

Each rank times its own replica; the whole job's throughput is both ranks' work
over the slower rank's time, and every rank agrees on it. Also checks a process
without a process group, and ranks read from torchrun's environment.
"""

import os
import socket

import pytest
import torch.multiprocessing as mp

from albedo_b200.replicas import Ranks, max_over_ranks, ranks_from_env, whole_job_throughput


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        ranks = ranks_from_env()
        local_ms = 400.0 + 150.0 * ranks.rank  # rank 1 is the slower replica
        slowest = max_over_ranks(local_ms, dist, "cpu")
        value = whole_job_throughput(33.1776, 5, ranks.world, slowest / 1e3)
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
            f.write(f"{ranks.rank} {ranks.world} {slowest} {value}\n")
    finally:
        dist.destroy_process_group()


def test_two_ranks_agree_on_the_slowest_time_and_the_whole_job_throughput(tmp_path):
    world = 2
    mp.spawn(rank_main, args=(world, free_port(), str(tmp_path)), nprocs=world, join=True)
    lines = [(tmp_path / f"rank{r}.txt").read_text().split() for r in range(world)]
    for r, (rank, w, slowest, value) in enumerate(lines):
        assert int(rank) == r and int(w) == world
        assert float(slowest) == 550.0
        assert float(value) == pytest.approx(2 * 33.1776 * 5 / 0.55)


def test_one_process_needs_no_process_group(monkeypatch):
    for key in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(key, raising=False)
    assert ranks_from_env() == Ranks(0, 1, 0)
    assert max_over_ranks(123.0) == 123.0
    assert whole_job_throughput(10.0, 3, 1, 2.0) == 15.0
    with pytest.raises(ValueError):
        whole_job_throughput(10.0, 3, 1, 0.0)
