"""Python twin of the reference's training driver (src/train.rs:14-105).

`train_files` makes the same C-ABI calls, in the same order, over the same
files as src/train.rs does (z.bin mapped read-write, w.bin/d.bin/k_d.bin
read-only, word counts from c.txt).  The compiled C++ twin of the same loop is
csrc/host/gpulda_train.cpp.
"""
from __future__ import annotations

import numpy as np

from . import GpuldaError, Sampler, corpus


def fill_sizes(d_len: np.ndarray, start: int, buffer_size: int, max_D: int) -> tuple[int, int]:
    """src/train.rs:20-47: documents are taken while the next length is
    nonzero and the buffer holds at most max_D documents and buffer_size
    tokens.  A document longer than buffer_size is fatal, as in the
    reference."""
    n_docs = n_tokens = 0
    i = start
    while True:
        size = int(d_len[i]) if i < len(d_len) else 0
        n_docs += 1
        n_tokens += size
        if size > buffer_size:
            raise GpuldaError(4, f"document size exceeded buffer size: {size}")
        if size == 0 or n_docs > max_D or n_tokens > buffer_size:
            return n_docs - 1, n_tokens - size
        i += 1


def iterate_buffers(z, w, d_len, k_d, buffer_size: int, max_D: int):
    """Yields (z, w, d, k_d) views buffer by buffer, as fill_buffer /
    empty_buffer walk the files (src/train.rs:20-58)."""
    doc = tok = 0
    while True:
        n_docs, n_tokens = fill_sizes(d_len, doc, buffer_size, max_D)
        if n_docs == 0:
            return
        yield (z[tok:tok + n_tokens], w[tok:tok + n_tokens], d_len[doc:doc + n_docs],
               k_d[doc:doc + n_docs] if k_d is not None else None)
        doc += n_docs
        tok += n_tokens


def train_files(paths: dict, K: int, alpha: float = 0.1, beta: float = 0.1, n_mc: int = 1,
                buffer_size: int = 33554432, max_D: int = 16384, seed: int = 0, flags: int = 0,
                on_iteration=None) -> None:
    """src/train.rs:60-105 over the reference's files (defaults from
    src/args.rs:17-59)."""
    counts = corpus.read_counts(paths["c"])
    z = np.memmap(paths["z"], dtype="<u4", mode="r+")
    w = np.memmap(paths["w"], dtype="<u4", mode="r")
    d = np.memmap(paths["d"], dtype="<u4", mode="r")
    k_d = np.memmap(paths["k_d"], dtype="<u4", mode="r")
    with Sampler(alpha, beta, K, counts, buffer_size=buffer_size, max_D=max_D, n_buffers=1, seed=seed,
                 flags=flags) as s:
        for it in range(n_mc):
            s.sample_phi()
            for zb, wb, db, kb in iterate_buffers(z, w, d, k_d, buffer_size, max_D):
                zc = np.ascontiguousarray(zb)
                s.sweep_buffer(0, zc, np.ascontiguousarray(wb), np.ascontiguousarray(db),
                               np.ascontiguousarray(kb))
                zb[:] = zc
            z.flush()
            if on_iteration is not None:
                on_iteration(it, s)
