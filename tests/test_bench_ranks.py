"""The multi-rank plumbing of bench.py on the CPU: two ranks over gloo (as
`bench.py --gpus 2` runs under torchrun, one process per GPU). Training does not
shard -- each rank is an independent replica -- so the only cross-rank steps are the
barriers around the timed region and the max over ranks of its duration; and under
torchrun the reference arm runs on rank 0 alone, the other ranks leaving at once."""
import argparse
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist

    import bench
    args = argparse.Namespace(impl="reference", gpus=world, steps=1, warmup=0)
    w, r, local = bench.dist_setup(args)  # gloo for the CPU arm
    assert (w, r, local) == (world, rank, rank)
    bench.barrier(w)
    # a rank's timed region: the job's time is the slowest rank's
    t = bench.max_over_ranks(1.0 + rank, w)
    printed = io.StringIO()
    if rank != 0:
        with redirect_stdout(printed):
            bench.run_reference(args, w, r)  # not rank 0: no work, no line
    bench.barrier(w)
    out.put((rank, t, printed.getvalue()))
    dist.destroy_process_group()


def test_two_ranks_gloo():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[1] for g in got] == [2.0, 2.0]  # max over ranks on every rank
    assert got[1][2] == ""  # rank 1 of the reference arm printed nothing
