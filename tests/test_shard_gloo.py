"""Document sharding's host logic on the CPU: two gloo ranks each sweep their
token-balanced range of documents (numbered from the range's first global
token) with the oracle and add their count tables after every iteration; the
chain must equal the single-process chain over the whole corpus bit for bit
(topics and counts) and its log-likelihood the sum of the ranks' parts."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from gpupolyaurnlda_b200.shard import shard_ranges

N_ITER = 3


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


class OracleShard:
    """CPU backend for ShardedChain: the oracle chain over one shard."""

    def __init__(self, c, shard):
        import oracle
        self.ch = oracle.Chain(c.K, c.alpha, c.beta, c.counts, seed=7, threads=1)
        self.z = c.z[shard.tok0:shard.tok1].copy()
        self.w = c.w[shard.tok0:shard.tok1]
        self.d = c.d_len[shard.doc0:shard.doc1]
        self.base = shard.tok0
        self.ll = 0.0

    def sweep(self):
        self.ch.sample_phi()
        self.ch.tok_base = self.base
        self.ll = self.ch.sweep(self.w, self.z, self.d, want_ll=True)["ll"]

    def counts(self):
        import torch
        return torch.from_numpy(self.ch.n.view(np.int32))

    def loglik(self):
        return self.ll


def _rank(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist

    from gpupolyaurnlda_b200 import corpus
    from gpupolyaurnlda_b200.shard import ShardedChain

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    c = corpus.generate("small", seed=2, D=300)
    sh = shard_ranges(c.d_len, world)[rank]
    be = OracleShard(c, sh)
    chain = ShardedChain(be)
    lls = [chain.iterate(1, want_ll=True) for _ in range(N_ITER)]
    out[rank] = (sh.tok0, be.z.copy(), be.ch.n.copy(), lls)
    dist.barrier()
    dist.destroy_process_group()


def test_shard_ranges_cover_and_balance():
    d = np.random.default_rng(0).integers(1, 50, 1000).astype(np.uint32)
    for world in (1, 2, 3, 8):
        sh = shard_ranges(d, world)
        assert sh[0].doc0 == 0 and sh[-1].doc1 == len(d) and sh[-1].tok1 == int(d.sum())
        assert all(a.doc1 == b.doc0 and a.tok1 == b.tok0 for a, b in zip(sh, sh[1:]))
        sizes = [s.tok1 - s.tok0 for s in sh]
        assert max(sizes) - min(sizes) <= 2 * int(d.max())


def test_two_rank_shards_equal_single_chain(oracle_lib):
    from gpupolyaurnlda_b200 import corpus
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    c = corpus.generate("small", seed=2, D=300)
    ch = oracle_lib.Chain(c.K, c.alpha, c.beta, c.counts, seed=7, threads=1)
    z = c.z.copy()
    lls = []
    for _ in range(N_ITER):
        ch.sample_phi()
        lls.append(ch.sweep(c.w, z, c.d_len, want_ll=True)["ll"])
    z_sh = np.concatenate([res[r][1] for r in range(world)])
    assert (z_sh == z).all()
    for r in range(world):
        assert (res[r][2] == ch.n).all()  # every rank holds the summed table
        np.testing.assert_allclose(res[r][3], lls, rtol=1e-9)
