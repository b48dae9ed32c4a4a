"""GPU parity of the large-K sweep against the CPU oracle, with each
document's topic counts in shared memory either as a sorted (topic, count)
list (the default) or in the order-preserving Robin Hood hash map
(GPULDA_FLAG_HASHMAP) -- src/cu/hashmap.cuh's role: topics and counts bit for
bit, through the resident-corpus and the buffer entry points, for short
documents (one launch) and long ones (a second launch sized for the
longest)."""
import dataclasses

import numpy as np
import pytest

import gpupolyaurnlda_b200 as g
from gpupolyaurnlda_b200 import corpus

pytestmark = pytest.mark.gpu


def _workload(K, V, D, lens=("lognormal", 4.2, 0.6, 5, 2000)):
    return dataclasses.replace(corpus.WORKLOADS["large_k10000"], K=K, V=V, D=D, doc_len=lens)


STORES = [0, g.GPULDA_FLAG_HASHMAP]


# (K, V, D, document lengths): the last case has documents of every launch
# tier -- at most 256 tokens, up to 1024, and longer
@pytest.mark.parametrize("store", STORES, ids=["pairs", "hashmap"])
@pytest.mark.parametrize("K,V,D,lens", [(4096, 3000, 3000, None), (10000, 2000, 1500, None),
                                        (4096, 2500, 500, ("lognormal", 6.0, 0.8, 5, 3000))])
def test_map_sweep_matches_oracle(gpu_lib, oracle_lib, K, V, D, lens, store):
    c = corpus.generate(_workload(K, V, D, **({"lens": lens} if lens else {})), seed=5, device="cuda")
    assert c.d_len.max() > 256 and c.d_len.min() <= 256  # both launches run
    if lens:
        assert c.d_len.max() > 1024 and ((c.d_len > 256) & (c.d_len <= 1024)).any()
    ch = oracle_lib.Chain(c.K, c.alpha, c.beta, c.counts, seed=3)
    z_orc = c.z.copy()
    with g.Sampler(c.alpha, c.beta, c.K, c.counts, buffer_size=16, max_D=4, seed=3,
                   flags=g.GPULDA_FLAG_LOGLIK | store) as s:
        s.corpus_load(c.z.copy(), c.w, c.d_len)
        for it in range(3):
            s.corpus_sweep(1)
            ch.sample_phi()
            r = ch.sweep(c.w, z_orc, c.d_len, want_ll=True)
            z = s.corpus_z()
            assert (z == z_orc).all(), f"iteration {it}: {(z != z_orc).sum()} topics differ"
            n = s.read_state(q=False, alias=False, A=False, S=False, nnz=False)["n"]
            assert (n == ch.n).all()
            ll, _ = s.loglik()
            assert abs(ll - r["ll"]) <= 1e-4 * abs(r["ll"])
    # the buffer entry point gives the same chain
    z_buf = c.z.copy()
    from gpupolyaurnlda_b200.train import iterate_buffers
    with g.Sampler(c.alpha, c.beta, c.K, c.counts, buffer_size=200000, max_D=700, seed=3, flags=store) as s:
        for _ in range(3):
            s.sample_phi()
            for zb, wb, db, kb in iterate_buffers(z_buf, c.w, c.d_len, c.k_d(), 200000, 700):
                s.sweep_buffer(0, zb, wb, db, kb)
    assert (z_buf == z_orc).all()


@pytest.mark.parametrize("store", STORES, ids=["pairs", "hashmap"])
def test_map_clustered_topics(gpu_lib, oracle_lib, store):
    """Documents whose topics are all distinct and packed at the top of the
    topic range: every insertion lands in one long run near the end of the
    table, the case the tail capacity is sized for."""
    K, V = 4096, 64
    rng = np.random.default_rng(9)
    lens = np.array([300, 256, 40, 1, 255, 600], np.uint32)
    z = np.concatenate([np.arange(K - L, K, dtype=np.uint32) if i % 2 == 0 else
                        rng.integers(0, K, L).astype(np.uint32) for i, L in enumerate(lens)])
    w = rng.integers(0, V, len(z)).astype(np.uint32)
    counts = np.bincount(w, minlength=V).astype(np.uint32) + 1
    order = np.argsort(-counts.astype(np.int64), kind="stable")
    counts = counts[order]
    z_gpu = z.copy()
    with g.Sampler(0.01, 0.05, K, counts, buffer_size=16, max_D=4, seed=1, flags=store) as s:
        s.corpus_load(z_gpu, w, lens)
        n0 = s.read_state(q=False, alias=False, A=False, S=False, nnz=False)["n"]
        s.corpus_sweep(1)
        z_gpu = s.corpus_z()
    phi = oracle_lib.phi_step(K, V, 0.05, n0, 0, 1, 0)
    z_orc = z.copy()
    oracle_lib.z_sweep(K, V, 0.01, phi, w, z_orc, lens, 0, key0=1)
    assert (z_gpu == z_orc).all()
