"""The multi-GPU plumbing of bench.py (one process per GPU, replicas only)
on the CPU: two gloo ranks initialise the process group the way bench.py
does under torchrun, meet at its barrier and agree on the maximum of their
step times, which is what the whole-job throughput is computed from."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
mp = pytest.importorskip("torch.multiprocessing")


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    import bench
    import torch.distributed as dist

    try:
        r, w, local = bench.dist_init(world, backend="gloo")
        bench.barrier(w)
        t = bench.max_over_ranks(10.0 * (r + 1), w)  # rank r's step time
        # whole-job throughput as bench.py reports it: units of all ranks / max time
        nbytes = 1000
        value = w * 4 * nbytes / (t / 1e3) / 1e9
        bench.barrier(w)
        q.put((r, w, local, t, value))
    finally:
        if dist.is_initialized():
            dist.destroy_process_group()


def test_two_gloo_ranks_max_over_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    got = sorted(q.get(timeout=5) for _ in range(world))
    assert [g[0] for g in got] == [0, 1]
    assert all(g[1] == world and g[2] == g[0] for g in got)
    assert all(g[3] == 20.0 for g in got)  # every rank sees the slowest rank's time
    assert got[0][4] == got[1][4] == pytest.approx(2 * 4 * 1000 / 0.020 / 1e9)
