"""Multi-rank host logic on CPU (gloo, 2 ranks): contiguous Sobol blocks per rank plus one
all_reduce give keldy's single-rank sums. Each rank's block is evaluated by the CPU
oracle here, standing in for that rank's GPU."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from keldy_b200 import parallel


def test_shard_covers_every_point_once():
    for n, world in [(10, 3), (4096, 8), (7, 7), (5, 8), (0, 2)]:
        blocks = [parallel.shard(n, r, world, k_first=11) for r in range(world)]
        ks = [k for k0, c in blocks for k in range(k0, k0 + c)]
        assert ks == list(range(11, 11 + n))
    with pytest.raises(ValueError):
        parallel.shard(10, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, golden_path, out):
    import torch.distributed as dist
    from oracle.pyoracle import Oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    g = np.load(golden_path)
    o = Oracle()
    m = o.model(10.0, g["table_beta20_lesser"], g["table_beta20_greater"])
    A, B = (10.0, 0, 0, 0, 0), (10.0, 0, 1, 0, 0)
    chain = [(1, 10.0, 0.0), (2, 10.0, 1.0)]
    sums = []
    for order, n in ((2, 301), (3, 257)):
        k0, cnt = parallel.shard(n, rank, world)
        s, npts, ndom, _ = o.integrate(m, A, B, chain, order, cnt, seed=k0 - 1)
        sums.append((s, npts, ndom))
    red = parallel.allreduce_sums(sums)
    if rank == 0:
        out.put(red)
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_equal_one(oracle, golden):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    path = os.path.join(os.path.dirname(__file__), "golden", "golden.npz")
    procs = [ctx.Process(target=_rank, args=(r, 2, port, path, q)) for r in range(2)]
    for p in procs:
        p.start()
    red = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    m = oracle.model(10.0, golden["table_beta20_lesser"], golden["table_beta20_greater"])
    for (order, n), (s, npts, ndom) in zip(((2, 301), (3, 257)), red):
        w, wn, wd, sc = oracle.integrate(m, (10.0, 0, 0, 0, 0), (10.0, 0, 1, 0, 0), [(1, 10.0, 0.0), (2, 10.0, 1.0)],
                                         order, n)
        assert (npts, ndom) == (wn, wd)
        assert abs(s - w) <= 1e-13 * sc
