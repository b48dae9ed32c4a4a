"""GPU parity at the benchmarked sizes: the CUDA library against the CPU
oracle on the full mid workload (K=1000, V=100,000, D=300,000, ~1.0e8 tokens)
and the full large workload (V=140,000, D=8,000,000, ~6.4e8 tokens) at
K=1000 and K=10000 (the sorted-pair-list store), and a fold-in of a 20,000-token
request against the full mid model.

Each sweep case runs the chain on the GPU for two iterations from random topics
(the corpus resident, as the benchmark runs it), then one more iteration
teacher-forced: the oracle starts from the GPU's counts and topics and must
give the same Phi step (fixed-point Phi, dense masses, per-topic normalisers,
nonzero counts, alias tables) bit for bit, the same topic for every token, the
same rebuilt counts and sparse-work counter, and the joint log-likelihood
within 1e-4 relative.  Reference semantics: src/cu/polyaurn.cu:87-123 (Phi
step), src/cu/topics.cu:36-105 (the sweep and the count rebuild)."""
import gc

import numpy as np
import pytest

import gpupolyaurnlda_b200 as g
from gpupolyaurnlda_b200 import corpus
from gpupolyaurnlda_b200.serve import Server, zipf_requests

pytestmark = pytest.mark.gpu

LL_RTOL = 1e-4
SEED, CHAIN = 3, 1


def _teacher_forced(c, oracle_lib, warm=2):
    with g.Sampler(c.alpha, c.beta, c.K, c.counts, buffer_size=16, max_D=4, seed=SEED, chain=CHAIN,
                   flags=g.GPULDA_FLAG_LOGLIK) as s:
        s.corpus_load(c.z.copy(), c.w, c.d_len)
        s.corpus_sweep(warm)
        n_prev = s.read_state(q=False, alias=False, A=False, S=False, nnz=False)["n"]
        z_prev = s.corpus_z()
        s.corpus_sweep(1)
        ll_gpu, skipped_gpu = s.loglik()
        work_gpu = s.counters()["sparse_work"]
        # Phi step of iteration `warm` from the GPU's counts
        phi = oracle_lib.phi_step(c.K, c.V, c.beta, n_prev, warm, SEED, CHAIN)
        del n_prev
        st = s.read_state(n=False)
        for k in ("q", "A", "S", "nnz"):
            assert (st[k] == phi[k]).all(), f"{k} differs from the oracle"
        nnz = phi["nnz"]
        live_g = oracle_lib.live_alias_entries(st.pop("alias"), nnz, c.K)
        live_o = oracle_lib.live_alias_entries(phi["alias"], nnz, c.K)
        assert (live_g == live_o).all(), "alias tables differ from the oracle"
        del live_g, live_o, st
        gc.collect()
        # the sweep of iteration `warm` from the GPU's topics
        z_gpu = s.corpus_z()
        n_gpu = s.read_state(q=False, alias=False, A=False, S=False, nnz=False)["n"]
    r = oracle_lib.z_sweep(c.K, c.V, c.alpha, phi, c.w, z_prev, c.d_len, warm, key0=SEED, key1=CHAIN, want_ll=True)
    bad = np.nonzero(z_gpu != z_prev)[0]
    assert len(bad) == 0, f"{len(bad)} of {c.n_tokens} topics differ from the oracle (first at token {bad[:5]})"
    assert (n_gpu == r["n"]).all(), "rebuilt counts differ from the oracle"
    assert int(r["stats"][2]) == work_gpu, "sparse-work counter differs from the oracle"
    assert r["ll_skipped"] == skipped_gpu
    assert abs(ll_gpu - r["ll"]) <= LL_RTOL * abs(r["ll"]), (ll_gpu, r["ll"])
    # size-independent properties of the rebuilt counts
    assert int(n_gpu.sum(dtype=np.uint64)) == c.n_tokens
    assert (n_gpu.reshape(c.V, c.K).sum(axis=1, dtype=np.uint64) == np.bincount(c.w, minlength=c.V)).all()
    return phi


@pytest.fixture(scope="module")
def mid(gpu_lib):
    return corpus.generate("mid", seed=1, device="cuda")


def test_mid_full_teacher_forced(mid, oracle_lib):
    _teacher_forced(mid, oracle_lib)


@pytest.mark.parametrize("workload", ["large_k1000", "large_k10000"])
def test_large_full_teacher_forced(gpu_lib, oracle_lib, workload):
    c = corpus.generate(workload, seed=1, device="cuda")
    assert c.n_docs == 8_000_000
    _teacher_forced(c, oracle_lib)
    del c
    gc.collect()


def test_fold_in_long_request_on_mid_model(mid, oracle_lib):
    """Fold-in against the full mid model (K=1000, V=100,000 after two
    training iterations): requests of 5 to 20,000 tokens, among them one of
    20,000, theta bit for bit and the log-likelihood within 1e-9 against the
    oracle's fold-in."""
    c = mid
    with g.Sampler(c.alpha, c.beta, c.K, c.counts, buffer_size=16, max_D=4, seed=SEED, chain=CHAIN) as s:
        s.corpus_load(c.z.copy(), c.w, c.d_len)
        s.corpus_sweep(2)
        st = s.read_state(n=False, S=False)
        srv = Server(8, seed=5, chain=1)
    try:
        lengths, words = zipf_requests(24, c.V, 77, mu=5.0, sigma=1.2, lo=5, hi=20000)
        lengths[0] = 20000
        lengths[1] = 5
        words = np.resize(words, int(lengths.sum())).astype(np.uint32)
        ids = np.arange(24, dtype=np.uint64) + np.uint64(1 << 33)
        srv.submit(ids, lengths, words)
        srv.drain()
        out = srv.poll(64)
        assert len(out["ids"]) == len(ids)
        order = np.argsort(out["ids"])
        ref = oracle_lib.fold_in(c.K, c.V, c.alpha, st, words, lengths, ids, 8, seed=5, chain=1)
        assert (out["theta"][order].view(np.uint32) == ref["theta"].view(np.uint32)).all()
        assert (out["skipped"][order] == ref["skipped"]).all()
        np.testing.assert_allclose(out["ll"][order], ref["ll"], rtol=1e-9, atol=1e-9)
    finally:
        srv.close()
