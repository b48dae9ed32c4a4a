"""Synthetic corpora from the LDA generative model, in the reference's formats.

The reference's preprocess step (src/preprocess.rs:16-72) writes
  z.bin   u32 per token, initial topic ~ Uniform{0..K-1}
  w.bin   u32 per token, word id
  d.bin   u32 per document, its length
  k_d.bin u32 per document, number of distinct initial topics
  c.txt   "token<TAB>id<TAB>count" per word, ids ranked by descending count
and its output step (src/output.rs:27-62) writes one line per document of
"token:topic<TAB>..." pairs.  This module produces the same files from seeded
synthetic data (no public dataset is involved) and reads them back.

Workloads (sizes of the benchmark's configurations):
  small   K=20, V=5000, D=2000, L ~ Poisson(100) (zeros redrawn),
          Phi_true[k] ~ Dir(0.01), theta ~ Dir(0.1), alpha=0.1, beta=0.01
  mid     K=1000, V=100000, D=300000, L = round(lognormal(5.5, 0.8)) clipped
          to [10, 5000]; topics Dir(0.01) times Zipf(1.05) weights over one
          random vocabulary permutation, renormalised; theta ~ Dir(0.1);
          alpha=50/K, beta=0.01
  large   K in {1000, 10000}, V=140000, D=8e6, L = lognormal(4.2, 0.6) clipped
          to [5, 2000], same topic generator
Dirichlet(a) with a << 1 is drawn in log space, G(a) = G(a+1) U^(1/a), to avoid
underflow.
"""
from __future__ import annotations

import dataclasses
import os

import numpy as np
import torch


@dataclasses.dataclass
class Workload:
    name: str
    K: int
    V: int
    D: int
    alpha: float
    beta: float
    doc_len: tuple  # ("poisson", mean) or ("lognormal", mu, sigma, lo, hi)
    zipf: float | None  # Zipf exponent of the vocabulary weights, None for plain Dirichlet
    topic_conc: float = 0.01
    doc_conc: float = 0.1


WORKLOADS = {
    "small": Workload("small", 20, 5000, 2000, 0.1, 0.01, ("poisson", 100.0), None),
    "mid": Workload("mid", 1000, 100000, 300000, 0.05, 0.01, ("lognormal", 5.5, 0.8, 10, 5000), 1.05),
    "large_k1000": Workload("large_k1000", 1000, 140000, 8000000, 0.05, 0.01, ("lognormal", 4.2, 0.6, 5, 2000), 1.05),
    "large_k10000": Workload("large_k10000", 10000, 140000, 8000000, 0.005, 0.01, ("lognormal", 4.2, 0.6, 5, 2000),
                             1.05),
}


@dataclasses.dataclass
class Corpus:
    K: int
    V: int
    alpha: float
    beta: float
    w: np.ndarray      # u32 tokens, word ids ranked by descending count
    z: np.ndarray      # u32 initial topics
    d_len: np.ndarray  # u32 document lengths
    counts: np.ndarray  # u32 per word id (descending)
    z_true: np.ndarray | None = None

    @property
    def n_tokens(self) -> int:
        return int(len(self.w))

    @property
    def n_docs(self) -> int:
        return int(len(self.d_len))

    def k_d(self) -> np.ndarray:
        """Distinct topics per document (src/preprocess.rs:66-68)."""
        doc = np.repeat(np.arange(self.n_docs, dtype=np.int64), self.d_len.astype(np.int64))
        key = np.unique(doc * self.K + self.z.astype(np.int64))
        return np.bincount(key // self.K, minlength=self.n_docs).astype(np.uint32)


def _log_dirichlet(shape, conc: float, gen: torch.Generator, device) -> torch.Tensor:
    """log of Dirichlet(conc * 1) rows (last dim), drawn in log space."""
    g1 = torch._standard_gamma(torch.full(shape, conc + 1.0, dtype=torch.float64, device=device), generator=gen)
    u = torch.rand(shape, dtype=torch.float64, device=device, generator=gen).clamp_min(1e-300)
    lg = torch.log(g1) + torch.log(u) / conc
    return lg - torch.logsumexp(lg, dim=-1, keepdim=True)


def _doc_lengths(wl: Workload, gen: torch.Generator, device) -> torch.Tensor:
    if wl.doc_len[0] == "poisson":
        L = torch.poisson(torch.full((wl.D,), wl.doc_len[1], dtype=torch.float64, device=device), generator=gen)
        while True:
            zero = L == 0
            if not bool(zero.any()):
                break
            L[zero] = torch.poisson(torch.full((int(zero.sum()),), wl.doc_len[1], dtype=torch.float64, device=device),
                                    generator=gen)
        return L.long()
    _, mu, sigma, lo, hi = wl.doc_len
    L = torch.exp(mu + sigma * torch.randn(wl.D, dtype=torch.float64, device=device, generator=gen))
    return torch.round(L).clamp(lo, hi).long()


def _inverse_cdf_rows(logp: torch.Tensor, row: torch.Tensor, gen: torch.Generator) -> torch.Tensor:
    """Samples one column per entry of `row` from the row's distribution
    (rows of exp(logp)); all rows share one sorted array offset by the row id."""
    R, Cn = logp.shape
    p = torch.exp(logp)
    cdf = torch.cumsum(p, dim=1)
    cdf = cdf / cdf[:, -1:]
    cdf = cdf + torch.arange(R, dtype=torch.float64, device=logp.device)[:, None]
    flat = cdf.reshape(-1)
    out = torch.empty_like(row)
    step = 1 << 24
    for s in range(0, len(row), step):
        r = row[s:s + step]
        u = torch.rand(len(r), dtype=torch.float64, device=logp.device, generator=gen)
        idx = torch.searchsorted(flat, r.double() + u, right=True).clamp_max(R * Cn - 1)
        out[s:s + step] = idx - r * Cn
    return out.clamp_(0, Cn - 1)


def generate(wl: Workload | str, seed: int = 1, device: str = "cpu", D: int | None = None) -> Corpus:
    """Draws a corpus; word ids are re-ranked by descending count and unused
    words dropped, as src/preprocess.rs:16-32 builds its vocabulary."""
    if isinstance(wl, str):
        wl = WORKLOADS[wl]
    if D is not None:
        wl = dataclasses.replace(wl, D=D)
    dev = torch.device(device)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    K, V = wl.K, wl.V
    L = _doc_lengths(wl, gen, dev)
    N = int(L.sum())
    doc = torch.repeat_interleave(torch.arange(wl.D, device=dev), L)
    # topic of each token from its document's theta
    z_true = torch.empty(N, dtype=torch.long, device=dev)
    chunk = max(1, (1 << 26) // K)
    starts = torch.cumsum(L, 0) - L
    for d0 in range(0, wl.D, chunk):
        d1 = min(wl.D, d0 + chunk)
        lt = _log_dirichlet((d1 - d0, K), wl.doc_conc, gen, dev)
        t0, t1 = int(starts[d0]), int(starts[d1 - 1] + L[d1 - 1])
        z_true[t0:t1] = _inverse_cdf_rows(lt, doc[t0:t1] - d0, gen)
    # words from the topics
    lphi = _log_dirichlet((K, V), wl.topic_conc, gen, dev)
    if wl.zipf is not None:
        perm = torch.randperm(V, generator=gen, device=dev)
        ranks = torch.empty(V, dtype=torch.float64, device=dev)
        ranks[perm] = torch.arange(1, V + 1, dtype=torch.float64, device=dev)
        lphi = lphi - wl.zipf * torch.log(ranks)[None, :]
        lphi = lphi - torch.logsumexp(lphi, dim=1, keepdim=True)
    w_raw = _inverse_cdf_rows(lphi, z_true, gen)
    del lphi
    # shuffle tokens within documents
    key = doc.double() + torch.rand(N, dtype=torch.float64, device=dev, generator=gen) * 0.5
    order = torch.argsort(key)
    w_raw, z_true = w_raw[order], z_true[order]
    # rank words by descending count; drop unused words
    cnt = torch.bincount(w_raw, minlength=V)
    order_w = torch.argsort(-cnt * (V + 1) + torch.arange(V, device=dev))  # count desc, id asc
    rank = torch.empty(V, dtype=torch.long, device=dev)
    rank[order_w] = torch.arange(V, device=dev)
    Vused = int((cnt > 0).sum())
    w = rank[w_raw]
    counts = cnt[order_w][:Vused]
    z0 = torch.randint(0, K, (N,), generator=gen, device=dev)
    to = lambda t: t.to(torch.int64).cpu().numpy().astype(np.uint32)
    return Corpus(K=K, V=Vused, alpha=wl.alpha, beta=wl.beta, w=to(w), z=to(z0), d_len=to(L), counts=to(counts),
                  z_true=to(z_true))


def batched_workloads(n: int = 64, seed: int = 1, D_scale: float = 1.0) -> list[Workload]:
    """The batched-chains workload: n independent problems with K drawn from
    {50, 200, 1000}, V from [5000, 50000], D from [1000, 100000] (times
    D_scale), document lengths lognormal(4.5, 1.0) clipped to [1, 65535] (the
    16-bit count width; the clip removes no mass at these parameters), the
    topic generator of ``mid``, alpha = 50/K, beta = 0.01.  Problem i is then
    drawn by ``generate(wl[i], seed=seed + 1000 + i)``."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        K = int(rng.choice([50, 200, 1000]))
        V = int(rng.integers(5000, 50001))
        D = max(1, int(round(int(rng.integers(1000, 100001)) * D_scale)))
        out.append(Workload(f"batch{i}", K, V, D, 50.0 / K, 0.01, ("lognormal", 4.5, 1.0, 1, 65535), 1.05))
    return out


# --- reference file formats ----------------------------------------------------

def write_files(c: Corpus, directory: str) -> dict:
    """Writes z.bin, w.bin, d.bin, k_d.bin, c.txt like src/preprocess.rs:42-72."""
    os.makedirs(directory, exist_ok=True)
    paths = {k: os.path.join(directory, f) for k, f in
             (("z", "z.bin"), ("w", "w.bin"), ("d", "d.bin"), ("k_d", "k_d.bin"), ("c", "c.txt"))}
    c.z.astype("<u4").tofile(paths["z"])
    c.w.astype("<u4").tofile(paths["w"])
    c.d_len.astype("<u4").tofile(paths["d"])
    c.k_d().astype("<u4").tofile(paths["k_d"])
    with open(paths["c"], "w") as f:
        for i, n in enumerate(c.counts):
            f.write(f"w{i}\t{i}\t{int(n)}\n")
    return paths


def read_counts(path: str) -> np.ndarray:
    """Third column of c.txt (src/train.rs:15-18)."""
    with open(path) as f:
        return np.array([int(line.rstrip("\n").split("\t")[2]) for line in f], dtype=np.uint32)


def read_names(path: str) -> dict:
    """id -> token from c.txt (src/output.rs:9-20)."""
    out = {}
    with open(path) as f:
        for line in f:
            tok, i = line.rstrip("\n").split("\t")[:2]
            out[int(i)] = tok
    return out


def write_output(z_path: str, w_path: str, d_path: str, c_path: str, out_path: str) -> None:
    """token:topic lines, one per document (src/output.rs:27-62)."""
    names = read_names(c_path)
    z = np.fromfile(z_path, dtype="<u4")
    w = np.fromfile(w_path, dtype="<u4")
    d = np.fromfile(d_path, dtype="<u4")
    pos = 0
    with open(out_path, "w") as f:
        for L in d:
            L = int(L)
            f.write("".join(f"{names[int(wi)]}:{int(zi)}\t" for wi, zi in zip(w[pos:pos + L], z[pos:pos + L])))
            f.write("\n")
            pos += L
