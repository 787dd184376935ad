"""The multi-GPU plumbing of bench.py (one process per GPU: a process group,
barriers, the max over ranks of the device times, one row shard per rank, the
reference arm on rank 0 only), run as two gloo ranks on the CPU."""
import argparse
import io
import os
import socket
from contextlib import redirect_stdout

import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist

    import bench

    r, w, _ = bench.dist_env()
    bench.init_dist(w, backend="gloo", timeout_s=60)
    slowest = bench.allreduce_max(10.0 + r, w)  # each rank's own time in, the slowest out
    bench.barrier(w)
    printed = ""
    if r == 1:  # the reference arm runs on rank 0 alone; other ranks leave without work
        buf = io.StringIO()
        with redirect_stdout(buf):
            bench.run_reference(argparse.Namespace(steps=1, warmup=0))
        printed = buf.getvalue()
    bench.barrier(w)
    dist.destroy_process_group()
    q.put((r, w, slowest, bench.shard_seed(r), printed))


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=180) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[0] for o in out] == [0, 1] and all(o[1] == 2 for o in out)
    assert all(o[2] == 11.0 for o in out)  # max over ranks, on every rank
    assert out[0][3] == 0 and out[0][3] != out[1][3]  # rank 0 holds the single-GPU rows; shards differ
    assert out[1][4] == ""  # rank 1 printed no reference line


def test_whole_job_throughput():
    import bench

    # rows of all ranks over the slowest rank's time
    assert bench.job_rows_per_s(1_000_000, 8, 10.0) == 8e8
    assert bench.job_rows_per_s(1_000_000, 1, 7.0) == 1_000_000 / 0.007
