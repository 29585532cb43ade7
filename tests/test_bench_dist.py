"""Host logic of bench.py's multi-GPU path on CPU: two gloo ranks check the
max-over-ranks timing reduction and the barrier, that each rank generates
its own file (one file per GPU, weak scaling), and that the reference arm
does its work on rank 0 only."""

from __future__ import annotations

import multiprocessing as mp
import os
import socket

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import datetime

    import torch.distributed as dist

    import bench
    from gpjson_b200 import datagen

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        r, w, _ = bench.dist_env()
        slowest = bench.max_over_ranks(10.0 + r, w)
        bench.barrier(w)
        head = bytes(datagen.tweets(4096, seed=datagen.SEED_BASE + 1 + r, p_empty_hashtags=0.3)[:256])
        args = bench.parse_args(["--impl", "reference", "--steps", "1", "--warmup", "0",
                                 "--cpu-sample", "65536"])
        if r != 0:
            bench.run_reference(args, r, w)  # returns at once: rank 0 alone runs the CPU arm
        out.put((r, slowest, head))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = [out.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got.sort()
    assert [g[1] for g in got] == [11.0, 11.0], "max over ranks"
    assert got[0][2] != got[1][2], "each rank indexes its own file"


def test_weak_scaling_value():
    """value = bytes of all ranks / slowest rank's time."""
    import bench

    assert bench.whole_job_gbs(1, 2 << 30, 10.0) == pytest.approx(214.748, rel=1e-4)
    assert bench.whole_job_gbs(4, 2 << 30, 10.0) == pytest.approx(4 * 214.748, rel=1e-4)
    args = bench.parse_args([])
    assert args.gpus == 1 and args.mode == "default" and args.warmup >= 3
    with pytest.raises(SystemExit):
        bench.parse_args(["--mode", "nonsense"])
