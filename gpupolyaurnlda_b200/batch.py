"""Batched chains: many independent LDA problems in one set of device arenas,
one CUDA graph per iteration (include/gpulda_batch.h).

The reference runs one model per process (src/cu/train.cu:16-29); a problem
here computes exactly what a solo ``Sampler`` with the same arguments, seed
and chain computes through ``corpus_load`` / ``corpus_sweep``.
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from . import BATCH_BUCKETS, BatchShape, GpuldaError, Problem, check, lib, GPULDA_FLAG_LOGLIK


@dataclasses.dataclass
class ProblemSpec:
    alpha: float
    beta: float
    K: int
    counts: np.ndarray   # V word counts
    z: np.ndarray        # initial topics
    w: np.ndarray        # word ids
    d_len: np.ndarray    # document lengths
    seed: int = 0
    chain: int = 0
    loglik: bool = True


class BatchChains:
    """Owner of one gpulda_batch handle."""

    def __init__(self, problems: list[ProblemSpec]):
        L = lib()
        L.gpulda_set_fatal_errors(0)
        self.h = None
        self.n = len(problems)
        self._keep = []
        arr = (Problem * self.n)()
        self.sizes = []
        for i, p in enumerate(problems):
            cnt = np.ascontiguousarray(p.counts, dtype=np.uint32)
            z = np.ascontiguousarray(p.z, dtype=np.uint32)
            w = np.ascontiguousarray(p.w, dtype=np.uint32)
            d = np.ascontiguousarray(p.d_len, dtype=np.uint32)
            self._keep += [cnt, z, w, d]
            arr[i] = Problem(alpha=p.alpha, beta=p.beta, K=p.K, V=len(cnt), C=cnt.ctypes.data, z=z.ctypes.data,
                             w=w.ctypes.data, d_len=d.ctypes.data, n_tokens=len(z), n_docs=len(d),
                             flags=GPULDA_FLAG_LOGLIK if p.loglik else 0, seed=p.seed, chain=p.chain)
            self.sizes.append((p.K, len(cnt), len(z)))
        h = C.c_void_p()
        check(L.gpulda_batch_create(arr, self.n, C.byref(h)), "gpulda_batch_create")
        self._keep = []  # the library copied everything it needs
        self.h = h

    def close(self) -> None:
        if self.h:
            lib().gpulda_batch_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sweep(self, n_iter: int = 1) -> None:
        check(lib().gpulda_batch_sweep(self.h, n_iter), "gpulda_batch_sweep")

    def sweep_async(self, n_iter: int, stream_handle: int) -> None:
        check(lib().gpulda_batch_sweep_async(self.h, n_iter, C.c_void_p(stream_handle)), "gpulda_batch_sweep_async")

    def sync(self) -> None:
        check(lib().gpulda_batch_sync(self.h), "gpulda_batch_sync")

    def z(self, p: int) -> np.ndarray:
        out = np.empty(self.sizes[p][2], np.uint32)
        check(lib().gpulda_batch_read_z(self.h, p, out.ctypes.data_as(C.POINTER(C.c_uint32))), "batch read_z")
        return out

    def counts(self, p: int) -> np.ndarray:
        K, V, _ = self.sizes[p]
        out = np.empty(K * V, np.uint32)
        check(lib().gpulda_batch_read_counts(self.h, p, out.ctypes.data_as(C.POINTER(C.c_uint32))),
              "batch read_counts")
        return out

    def loglik(self) -> tuple[np.ndarray, np.ndarray]:
        ll = np.zeros(self.n, np.float64)
        sk = np.zeros(self.n, np.uint64)
        check(lib().gpulda_batch_loglik(self.h, ll.ctypes.data_as(C.POINTER(C.c_double)),
                                        sk.ctypes.data_as(C.POINTER(C.c_uint64))), "batch loglik")
        return ll, sk

    def shapes(self) -> list[tuple[int, int, int]]:
        arr = (BatchShape * BATCH_BUCKETS)()
        check(lib().gpulda_batch_get_shapes(self.h, arr), "batch get_shapes")
        return [(s.z_warps_per_block, s.z_blocks_per_sm, s.phi_cells_per_block) for s in arr]

    def set_shapes(self, shapes: list[tuple[int, int, int]]) -> None:
        arr = (BatchShape * BATCH_BUCKETS)()
        for i, (a, b, c) in enumerate(shapes):
            arr[i] = BatchShape(a, b, c, 0)
        check(lib().gpulda_batch_set_shapes(self.h, arr), "batch set_shapes")

    def set_mode(self, mode: int, shape: tuple[int, int, int] | None = None) -> None:
        """BATCH_PER_BUCKET, BATCH_MERGED (one launch per stage over every
        problem) or BATCH_MERGED_SWEEP (per-bucket Phi step, one z sweep over
        every problem); `shape` sets the merged launches' (z warps per block,
        z blocks per SM, Poisson cells per block)."""
        sh = BatchShape(shape[0], shape[1], shape[2], 0) if shape else None
        check(lib().gpulda_batch_set_mode(self.h, mode, C.byref(sh) if sh else None), "batch set_mode")

    def tune(self, cache_path: str | None = None) -> int:
        n = C.c_uint32(0)
        check(lib().gpulda_batch_tune(self.h, cache_path.encode() if cache_path else None, C.byref(n)),
              "batch tune")
        return int(n.value)

    def info(self) -> dict:
        out = (C.c_uint64 * 9)()
        m = lib().gpulda_batch_info(self.h, out, 9)
        keys = ("problems", "tokens", "docs", "words", "cells", "device_bytes", "buckets", "iterations", "mode")
        return {k: int(out[i]) for i, k in enumerate(keys[:m])}


BATCH_PER_BUCKET, BATCH_MERGED, BATCH_MERGED_SWEEP = 0, 1, 2

__all__ = ["BatchChains", "ProblemSpec", "GpuldaError", "BATCH_PER_BUCKET", "BATCH_MERGED", "BATCH_MERGED_SWEEP"]
