"""Host side of `bench.py --gpus N` (N independent replicas, one process per
GPU) on CPU: two gloo ranks set up the process group the way the bench does,
take the max of their step times over ranks, pass the barrier on both sides
of the timed region and tear down.  The replicas exchange nothing else."""

import os
import socket
import sys
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, str(ROOT))
    import bench

    r, w, local = bench.dist_setup("gloo")
    bench.barrier()
    ms = 10.0 + 5.0 * r  # rank 1 is the slow one
    m = bench.max_over_ranks(ms)
    bench.barrier()
    import torch.distributed as dist

    if dist.is_initialized():
        dist.destroy_process_group()
    out.put((r, w, local, m))


def test_two_gloo_replicas_agree_on_the_max_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    codes = [p.exitcode for p in procs]
    for p in procs:
        if p.is_alive():
            p.kill()
    assert codes == [0, 0], codes
    got = sorted(q.get(timeout=5) for _ in range(2))
    assert got == [(0, 2, 0, 15.0), (1, 2, 1, 15.0)]


def test_single_process_needs_no_group():
    sys.path.insert(0, str(ROOT))
    import bench

    env = {k: os.environ.pop(k) for k in ("WORLD_SIZE", "RANK") if k in os.environ}
    try:
        assert bench.dist_setup("gloo") == (0, 1, 0)
        assert bench.max_over_ranks(3.5) == 3.5
    finally:
        os.environ.update(env)
