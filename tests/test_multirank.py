"""Host logic of the N > 1 bench path on CPU: two gloo ranks, each with its own parameter set (weak
scaling by parameter sets, no data-path collective), step time reduced as the max over ranks."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    r, w, _ = bench.rank_info()
    c = bench.workload(seed_offset=r, res=8, nsamples=16)
    m = bench.max_over_ranks(10.0 + r)
    q.put((r, w, float(c["params"].sum()), m))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, w0, s0, m0), (r1, w1, s1, m1) = out
    assert (r0, r1, w0, w1) == (0, 1, 2, 2)
    assert s0 != s1                       # each rank renders its own parameter set
    assert m0 == m1 == 11.0               # max over ranks
