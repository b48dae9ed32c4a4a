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


def model_requests(q: np.ndarray, K: int, n: int, seed: int, doc_conc: float = 0.1, mu: float = 5.0,
                   sigma: float = 1.2, lo: int = 5, hi: int = 20000, device: str = "cuda"):
    """Synthetic requests drawn from a model's own topics (the LDA generative
    process): per document theta ~ Dirichlet(doc_conc), lengths
    round(lognormal(mu, sigma)) clipped to [lo, hi], each token's topic from
    theta and its word from that topic's Phi column, Phi[k][w] =
    q[w][k] / sum_w q[w][k] (q: the V x K word-major fixed-point Phi).
    Returns (lengths u32, words u32)."""
    import torch
    rng = np.random.default_rng(seed)
    V = len(q) // K
    lengths = np.clip(np.round(rng.lognormal(mu, sigma, n)), lo, hi).astype(np.uint32)
    theta = rng.dirichlet(np.full(K, doc_conc), n)
    z = np.concatenate([rng.choice(K, int(L), p=th / th.sum()) for L, th in zip(lengths, theta)]).astype(np.int64)
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    qt = torch.from_numpy(np.ascontiguousarray(q, np.uint32).view(np.int32)).to(device).view(V, K)
    words = np.empty(len(z), np.uint32)
    zt = torch.from_numpy(z).to(device)
    order = torch.argsort(zt)
    zs = zt[order]
    bounds = torch.searchsorted(zs, torch.arange(K + 1, device=device)).cpu().numpy()
    out = torch.empty(len(z), dtype=torch.int64, device=device)
    for k0 in range(0, K, 64):  # topic columns in blocks: a K x V float64 table is not needed at once
        k1 = min(K, k0 + 64)
        col = (qt[:, k0:k1].to(torch.int64) & 0xffffffff).to(torch.float64).t()  # (k1-k0) x V
        cdf = torch.cumsum(col, dim=1)
        tot = cdf[:, -1:].clamp_min(1.0)
        cdf = cdf / tot + torch.arange(k1 - k0, device=device, dtype=torch.float64)[:, None]
        flat = cdf.reshape(-1)
        a, b = int(bounds[k0]), int(bounds[k1])
        if b > a:
            kk = zs[a:b] - k0
            u = torch.rand(b - a, dtype=torch.float64, device=device, generator=g)
            idx = torch.searchsorted(flat, kk.double() + u, right=True).clamp_max(flat.numel() - 1)
            out[order[a:b]] = (idx - kk * V).clamp_(0, V - 1)
    words[:] = out.cpu().numpy().astype(np.uint32)
    return lengths, words


def split_halves(lengths: np.ndarray, words: np.ndarray):
    """Document completion: the first ceil(L/2) tokens of every document are
    folded in, the rest are scored.  Returns (first lengths, first words,
    second lengths, second words)."""
    lengths = np.asarray(lengths, np.int64)
    first = (lengths + 1) // 2
    offs = np.concatenate([[0], np.cumsum(lengths)])
    in_first = np.arange(offs[-1]) - np.repeat(offs[:-1], lengths) < np.repeat(first, lengths)
    return (first.astype(np.uint32), np.ascontiguousarray(words[in_first], np.uint32),
            (lengths - first).astype(np.uint32), np.ascontiguousarray(words[~in_first], np.uint32))


def completion_loglik(q: np.ndarray, K: int, theta: np.ndarray, lengths: np.ndarray, words: np.ndarray,
                      device: str = "cuda") -> tuple[float, int]:
    """Held-out log-likelihood of document completion: sum over every scored
    token i of document d of log sum_k theta[d][k] Phi[k][w_i], with Phi[k][w]
    = q[w][k] / 2^32 (the fixed-point Phi the fold-in used).  theta is
    n x K (float), lengths/words the scored tokens.  Returns (sum, tokens
    scored); tokens whose mixture is zero are not scored."""
    import torch
    V = len(q) // K
    qt = torch.from_numpy(np.ascontiguousarray(q, np.uint32).view(np.int32)).to(device).view(V, K)
    th = torch.from_numpy(np.ascontiguousarray(theta, np.float32)).to(device).double()
    doc = torch.from_numpy(np.repeat(np.arange(len(lengths)), np.asarray(lengths, np.int64))).to(device)
    wt = torch.from_numpy(np.asarray(words, np.int64)).to(device)
    total, scored = 0.0, 0
    for a in range(0, len(wt), 1 << 16):
        rows = (qt[wt[a:a + (1 << 16)]].to(torch.int64) & 0xffffffff).double() / 4294967296.0
        p = (rows * th[doc[a:a + (1 << 16)]]).sum(dim=1)
        ok = p > 0
        total += float(torch.log(p[ok]).sum())
        scored += int(ok.sum())
    return total, scored


__all__ = ["Server", "zipf_requests", "model_requests", "split_halves", "completion_loglik"]
