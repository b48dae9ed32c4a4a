"""The multi-GPU form is independent chains, one per rank (the sampler's only
exchange, the count table, is per chain).  This runs that path's host logic
with two gloo ranks on the CPU: each rank runs its own chain (Philox key word
1 = rank) with the oracle, the job time is the max over ranks, and the value
is the whole-job rate bench.py reports."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import datetime
    import time

    import torch
    import torch.distributed as dist

    import bench
    import oracle
    from gpupolyaurnlda_b200 import corpus

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    c = corpus.generate("small", seed=1, D=100)
    ch = oracle.Chain(c.K, c.alpha, c.beta, c.counts, seed=0, chain=rank, threads=1)
    z = c.z.copy()
    t0 = time.perf_counter()
    for _ in range(2):
        ch.sample_phi()
        ch.sweep(c.w, z, c.d_len)
    local = time.perf_counter() - t0 + 0.05 * rank
    mx = bench.max_over_ranks(local, "cpu")
    zs = [torch.zeros(len(z), dtype=torch.int64) for _ in range(world)]
    dist.all_gather(zs, torch.from_numpy(z.astype(np.int64)))
    out[rank] = (local, mx, bench.replica_value(c.n_tokens, 2, world, mx),
                 float((zs[0] != zs[1]).float().mean()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_replicas():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    locals_ = [res[r][0] for r in range(world)]
    for r in range(world):
        assert res[r][1] == max(locals_)
        assert res[r][2] > 0
    assert res[0][3] > 0.3  # the two chains are different chains
