"""Fold-in serving with continuous batching (include/gpulda_serve.h).

A ``Server`` holds a fixed model on the device and estimates the topic
mixtures of incoming documents: ``submit`` queues requests, ``progress``
retires finished launches and launches queued requests as device memory and
launch slots free up, ``poll`` returns finished results.  The reference has no
serving path; its closest cousin is the z sweep without the count rebuild
(src/cu/topics.cu:36-105).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import SERVE_LAUNCH, SERVE_PERSISTENT, ServeArgs, check, lib

_U32P = C.POINTER(C.c_uint32)
_U64P = C.POINTER(C.c_uint64)


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


class Server:
    """Owner of one gpulda_serve handle.  ``q`` (V*K fixed-point Phi) builds
    the model from host data; without it the current single model of the
    library (a ``Sampler`` after at least one Phi step) is copied.  ``mode``
    "persistent" (resident warps take requests as they free up; ``slots`` =
    warps per SM) or "launch" (batches of up to ``max_batch`` per launch on
    ``slots`` streams; ``max_batch=1`` is one launch per document)."""

    def __init__(self, n_iter: int = 50, *, mode: str = "persistent", slots: int = 0, max_batch: int = 0,
                 max_inflight: int = 0, seed: int = 0, chain: int = 0, pool_bytes: int = 0,
                 q: np.ndarray | None = None, K: int | None = None, alpha: float | None = None):
        L = lib()
        L.gpulda_set_fatal_errors(0)
        self.h = None
        m = {"persistent": SERVE_PERSISTENT, "launch": SERVE_LAUNCH}[mode]
        a = ServeArgs(n_iter, m, slots, max_batch, max_inflight, chain, seed, pool_bytes)
        h = C.c_void_p()
        if q is None:
            check(L.gpulda_serve_create(C.byref(a), C.byref(h)), "gpulda_serve_create")
        else:
            q = np.ascontiguousarray(q, np.uint32).reshape(-1)
            check(L.gpulda_serve_create_from_phi(C.byref(a), K, len(q) // K, alpha, _p(q, C.c_uint32), C.byref(h)),
                  "gpulda_serve_create_from_phi")
        self.h = h
        st = self.stats()
        self.K, self.V = st["K"], st["V"]

    def close(self) -> None:
        if self.h:
            lib().gpulda_serve_destroy(self.h)
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

    def submit(self, ids, lengths, words) -> None:
        ids = np.ascontiguousarray(ids, np.uint64)
        lengths = np.ascontiguousarray(lengths, np.uint32)
        words = np.ascontiguousarray(words, np.uint32)
        check(lib().gpulda_serve_submit(self.h, len(ids), _p(ids, C.c_uint64), _p(lengths, C.c_uint32),
                                        _p(words, C.c_uint32)), "gpulda_serve_submit")

    def progress(self) -> None:
        check(lib().gpulda_serve_progress(self.h), "gpulda_serve_progress")

    def drain(self) -> None:
        check(lib().gpulda_serve_drain(self.h), "gpulda_serve_drain")

    def poll(self, max_n: int = 1 << 16, theta: bool = True) -> dict:
        ids = np.empty(max_n, np.uint64)
        th = np.empty((max_n, self.K), np.float32) if theta else None
        ll = np.empty(max_n, np.float64)
        sk = np.empty(max_n, np.uint32)
        done = np.empty(max_n, np.uint64)
        n = C.c_uint32(0)
        check(lib().gpulda_serve_poll(self.h, max_n, _p(ids, C.c_uint64),
                                      _p(th, C.c_float) if theta else None, _p(ll, C.c_double),
                                      _p(sk, C.c_uint32), _p(done, C.c_uint64), C.byref(n)), "gpulda_serve_poll")
        k = n.value
        return {"ids": ids[:k], "theta": th[:k] if theta else None, "ll": ll[:k], "skipped": sk[:k],
                "done_ns": done[:k]}

    def stats(self) -> dict:
        out = (C.c_uint64 * 10)()
        m = lib().gpulda_serve_stats(self.h, out, 10)
        keys = ("queued", "inflight", "ready", "launches", "finished", "pool_bytes", "pool_used", "deferred", "K",
                "V")
        return {k: int(out[i]) for i, k in enumerate(keys[:m])}


def zipf_requests(n: int, V: int, seed: int, mu: float = 5.0, sigma: float = 1.2, lo: int = 5, hi: int = 20000,
                  s: float = 1.05):
    """Synthetic requests: lengths round(lognormal(mu, sigma)) clipped to
    [lo, hi]; tokens Zipf(s) over word ids 0..V-1 (ids ranked by frequency, as
    the training vocabulary is)."""
    rng = np.random.default_rng(seed)
    lengths = np.clip(np.round(rng.lognormal(mu, sigma, n)), lo, hi).astype(np.uint32)
    p = 1.0 / np.arange(1, V + 1, dtype=np.float64) ** s
    cdf = np.cumsum(p)
    cdf /= cdf[-1]
    words = np.searchsorted(cdf, rng.random(int(lengths.sum())), side="right").clip(0, V - 1).astype(np.uint32)
    return lengths, words


__all__ = ["Server", "zipf_requests"]
