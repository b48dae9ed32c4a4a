"""Document sharding on the GPU (include/gpulda.h, gpulda_set_token_offset /
gpulda_count_table): a buffer swept out of order with its global token offset
gives the in-order chain bit for bit, and a one-rank NCCL ShardedChain over the
library's device count table gives the plain corpus chain.  (Two ranks need two
GPUs; their host logic runs with gloo in tests/test_shard_gloo.py.)"""
import socket

import numpy as np
import pytest

import gpupolyaurnlda_b200 as g
from gpupolyaurnlda_b200 import corpus
from gpupolyaurnlda_b200.shard import LibraryShard, ShardedChain, shard_ranges

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_token_offset_makes_buffer_order_irrelevant(gpu_lib):
    c = corpus.generate("small", seed=4, D=400)
    A, B = shard_ranges(c.d_len, 2)
    kd = c.k_d()
    runs = []
    for reverse in (False, True):
        z = c.z.copy()
        with g.Sampler(c.alpha, c.beta, c.K, c.counts, buffer_size=c.n_tokens, max_D=c.n_docs, seed=3) as s:
            for _ in range(3):
                s.sample_phi()
                parts = [B, A] if reverse else [A, B]
                for sh in parts:
                    if reverse:
                        s.set_token_offset(sh.tok0)
                    zb = z[sh.tok0:sh.tok1]  # a view: the sweep writes the topics back into z
                    s.sweep_buffer(0, zb, c.w[sh.tok0:sh.tok1], c.d_len[sh.doc0:sh.doc1], kd[sh.doc0:sh.doc1])
                if reverse:
                    s.set_token_offset(0)
            n = s.read_state(q=False, alias=False, A=False, S=False, nnz=False)["n"]
        runs.append((z, n))
    assert (runs[0][0] == runs[1][0]).all()
    assert (runs[0][1] == runs[1][1]).all()


def test_one_rank_nccl_sharded_chain_equals_plain_chain(gpu_lib):
    import datetime

    import torch
    import torch.distributed as dist

    c = corpus.generate("small", seed=5, D=300)
    with g.Sampler(c.alpha, c.beta, c.K, c.counts, buffer_size=16, max_D=4, seed=1,
                   flags=g.GPULDA_FLAG_LOGLIK) as s:
        s.corpus_load(c.z.copy(), c.w, c.d_len)
        for _ in range(3):
            s.corpus_sweep(1)
        z_plain = s.corpus_z()
        n_plain = s.read_state(q=False, alias=False, A=False, S=False, nnz=False)["n"]
        ll_plain = s.loglik()[0]
        assert (s.count_table().cpu().numpy().view(np.uint32) == n_plain.reshape(-1)).all()
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        with g.Sampler(c.alpha, c.beta, c.K, c.counts, buffer_size=16, max_D=4, seed=1,
                       flags=g.GPULDA_FLAG_LOGLIK) as s:
            chain = ShardedChain(LibraryShard(s, c.z, c.w, c.d_len, shard_ranges(c.d_len, 1)[0]))
            ll = None
            for _ in range(3):
                ll = chain.iterate(1, want_ll=True)
            assert (s.corpus_z() == z_plain).all()
            assert (s.read_state(q=False, alias=False, A=False, S=False, nnz=False)["n"] == n_plain).all()
            assert abs(ll - ll_plain) <= 1e-9 * abs(ll_plain)
    finally:
        dist.destroy_process_group()
