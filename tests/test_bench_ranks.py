"""The multi-rank path of bench.py on the CPU: world_size 2 over gloo.
Each rank runs its own replica of the step (no data-path collective); the
ranks' step times are combined as their maximum, so the whole-job rate is
ranks / slowest time.  Checked here with per-rank times the ranks know."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        ms = 1.0 + rank * 0.5                      # rank 1 is the slower one
        mx = bench.max_over_ranks(ms, dist, device="cpu")
        out[rank] = (mx, ws / (mx * 1e-3))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_two_ranks():
    import torch.multiprocessing as mp
    ws = 2
    port = _free_port()
    with mp.Manager() as man:
        out = man.dict()
        mp.spawn(_rank, args=(ws, port, out), nprocs=ws, join=True)
        res = dict(out)
    assert set(res) == {0, 1}
    for r in range(ws):
        mx, rate = res[r]
        assert mx == pytest.approx(1.5)
        assert rate == pytest.approx(2 / 1.5e-3)


def test_max_over_ranks_without_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(2.25) == 2.25
