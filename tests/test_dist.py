"""Multi-process host logic of the replica benchmark, on CPU with gloo
(world size 2): the timing reduction takes the max over ranks and every rank
takes the same collective steps."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank: int, world: int, port: int, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import datetime

    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world)
        mx = bench.allreduce_max(10.0 + rank, world)
        bench.barrier(world)
        q.put((rank, mx))
    finally:
        dist.destroy_process_group()


def test_replica_timing_is_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    got = dict(q.get(timeout=5) for _ in range(2))
    assert got == {0: 11.0, 1: 11.0}


def test_single_process_helpers():
    import bench

    assert bench.allreduce_max(3.5, 1) == 3.5
    bench.barrier(1)
    cfg = bench.config_dict(50000)
    assert cfg["grid"] == 1024 and cfg["slices_per_step"] == 100
    peak, kind = bench.measured_peaks()
    assert peak > 1000 and kind in ("measured", "fallback")


def test_clock_sampler_parses_reasons():
    import bench

    c = bench.ClockSampler(0)
    c.proc = type("P", (), {"terminate": lambda self: None, "wait": lambda self, timeout=None: 0})()
    c.lines = ["0, 1800, 1965, 700.0, 0x0, Not Active, Not Active, Not Active, Active",
               "0, 1830, 1965, 720.0, 0x0, Not Active, Not Active, Not Active, Not Active"]
    out = c.stop()
    assert out["sm_mhz"] == pytest.approx(1815.0)
    assert out["sm_max_mhz"] == 1965.0
    assert out["reasons"] == ["sw_power_cap"]
