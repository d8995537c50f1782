"""The multi-process plumbing of bench.py on CPU: two gloo ranks agree on
the maximum of their timed regions and on the whole-job rate, and the
reference arm's non-zero ranks leave without work (as under torchrun)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = [12.5, 20.0][rank]
    m = bench.reduce_max(ms, dist)
    rate = bench.whole_job_rate(world, 90, m)
    dist.barrier()
    dist.destroy_process_group()
    with open(os.path.join(out, f"r{rank}"), "w") as f:
        f.write(f"{m} {rate}")


def test_two_gloo_ranks_agree_on_the_max(tmp_path):
    port = _free_port()
    mp.start_processes(_rank, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    vals = [open(tmp_path / f"r{r}").read().split() for r in range(2)]
    for m, rate in vals:
        assert float(m) == 20.0
        assert abs(float(rate) - 2 * 90 / 0.020) < 1e-9


def test_reference_arm_nonzero_rank_exits_without_work(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--gpus", "2"])
    assert bench.main() == 0


def test_single_process_reduce_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_max(3.5, None) == 3.5
    assert bench.whole_job_rate(1, 30, 100.0) == pytest.approx(300.0)
