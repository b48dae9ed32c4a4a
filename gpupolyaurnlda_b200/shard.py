"""Document-sharded chains across processes (one GPU each).

Every rank holds the whole model and sweeps a contiguous range of documents
with about equal token counts.  The exchange is the count table: after each
iteration's sweeps the ranks add their tables in place (an all-reduce sum over
NCCL), so every rank's next Phi step starts from the same counts and the chain
equals the single-process chain bit for bit (include/gpulda.h: token offsets).
The reference runs one GPU (src/cu/train.cu); this is the natural partition of
its z sweep, whose documents are independent given Phi.
"""
from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass
class Shard:
    doc0: int
    doc1: int
    tok0: int
    tok1: int


def shard_ranges(d_len: np.ndarray, world: int) -> list[Shard]:
    """Contiguous document ranges with about equal token counts, one per rank
    (rank r ends after the first document whose running total reaches
    (r + 1) / world of the tokens)."""
    cum = np.concatenate([[0], np.cumsum(np.asarray(d_len, dtype=np.int64))])
    total = int(cum[-1])
    out, d0 = [], 0
    for r in range(world):
        if r == world - 1:
            d1 = len(d_len)
        else:
            d1 = int(np.searchsorted(cum, (total * (r + 1) + world - 1) // world, side="left"))
            d1 = max(d0, min(len(d_len), d1))
        out.append(Shard(d0, d1, int(cum[d0]), int(cum[d1])))
        d0 = d1
    return out


class ShardedChain:
    """One rank's part of a document-sharded chain.

    ``backend`` runs this rank's iterations: ``sweep()`` does one Phi step and
    one z sweep over the rank's documents (their tokens numbered from the
    shard's first global token), ``counts()`` returns the count table as a
    tensor sharing its memory, ``loglik()`` the rank's part of the joint
    log-likelihood.  ``Sampler`` with a loaded shard is the GPU backend
    (``LibraryShard``)."""

    def __init__(self, backend, group=None):
        self.backend = backend
        self.group = group

    def iterate(self, n_iter: int = 1, want_ll: bool = False):
        import torch
        import torch.distributed as dist
        ll = None
        for _ in range(n_iter):
            self.backend.sweep()
            n = self.backend.counts()
            dist.all_reduce(n, op=dist.ReduceOp.SUM, group=self.group)
            if n.is_cuda:
                torch.cuda.synchronize()
            if want_ll:
                t = torch.tensor([self.backend.loglik()], dtype=torch.float64, device=n.device)
                dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
                ll = float(t.item())
        return ll


class LibraryShard:
    """GPU backend: a ``Sampler`` holding the whole model and this rank's
    documents (corpus mode)."""

    def __init__(self, sampler, z, w, d_len, shard: Shard):
        self.s = sampler
        self.s.set_token_offset(shard.tok0)
        self.s.corpus_load(np.ascontiguousarray(z[shard.tok0:shard.tok1]), w[shard.tok0:shard.tok1],
                           d_len[shard.doc0:shard.doc1])
        self._n = None

    def sweep(self):
        self.s.corpus_sweep(1)

    def counts(self):
        if self._n is None:
            self._n = self.s.count_table()
        return self._n

    def loglik(self):
        return self.s.loglik()[0]


__all__ = ["Shard", "shard_ranges", "ShardedChain", "LibraryShard"]
