"""GPU parity: the CUDA library (through its C ABI) against the CPU oracle.

Counts, Phi, alias tables and topic assignments are compared bit for bit;
the joint log-likelihood within 1e-4 relative.  Inputs are seeded synthetic
corpora of the small workload (K=20, V~3300, D=2000, ~200k tokens) and
reduced slices of the mid workload.
"""
import numpy as np
import pytest

import gpupolyaurnlda_b200 as g

pytestmark = pytest.mark.gpu

LL_RTOL = 1e-4
TWO32 = 4294967296


def test_device_philox_published_vectors(gpu_lib, oracle_lib):
    ctr = np.array([[0, 0, 0, 0], [0xffffffff] * 4, [0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344]], np.uint32)
    keys = [(0, 0), (0xffffffff, 0xffffffff), (0xa4093822, 0x299f31d0)]
    want = [[0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8],
            [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd],
            [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]]
    for c, (k0, k1), w in zip(ctr, keys, want):
        assert g.device_philox(c, k0, k1)[0].tolist() == w
    rng = np.random.default_rng(0)
    ctr = rng.integers(0, 2 ** 32, (4096, 4), dtype=np.uint64).astype(np.uint32)
    assert (g.device_philox(ctr, 123, 456) == oracle_lib.philox(ctr, 123, 456)).all()


def _model(K=20, V=50, beta=0.01, alpha=0.1, **kw):
    counts = np.arange(V, 0, -1).astype(np.uint32) * 10
    return g.Sampler(alpha, beta, K, counts, **kw)


@pytest.mark.parametrize("beta", [0.01, 0.1, 0.0])
def test_device_tables_equal_oracle(gpu_lib, oracle_lib, beta):
    with _model(beta=beta) as s:
        cdf, lfac = s.tables()
    ocdf, _, olfac = oracle_lib.tables(beta)
    assert (cdf == ocdf).all()
    assert (lfac == olfac).all()


def test_device_poisson_matches_oracle(gpu_lib, oracle_lib):
    rng = np.random.default_rng(1)
    counts = np.concatenate([np.arange(0, 200), rng.integers(0, 64, 20000), rng.integers(64, 5000, 20000),
                             rng.integers(5000, 10 ** 7, 5000)]).astype(np.uint32)
    idx = rng.integers(0, 2 ** 40, len(counts), dtype=np.uint64)
    with _model(beta=0.01) as s:
        for t, stream, k0, k1 in [(0, 2, 0, 0), (7, 1, 99, 3)]:
            got = s.poisson(counts, idx, t, stream, k0, k1)
            want = oracle_lib.poisson(counts, idx, 0.01, t, stream, k0, k1)
            bad = np.nonzero(got != want)[0]
            assert len(bad) == 0, (counts[bad[:5]], got[bad[:5]], want[bad[:5]])
    # moments for the rejection branch
    lam = 1000
    x = oracle_lib.poisson(np.full(200000, lam, np.uint32), np.arange(200000, dtype=np.uint64), 0.01, 0, 2)
    assert abs(x.mean() - lam) < 0.5 and abs(x.var() / lam - 1) < 0.02


@pytest.mark.parametrize("K", [1, 2, 5, 20, 100, 1000, 5000, 11000])
def test_device_alias_matches_oracle(gpu_lib, oracle_lib, K):
    rng = np.random.default_rng(K)
    for dens in (1.0, 0.25, 0.01):
        q = (rng.integers(0, 2 ** 32, K, dtype=np.uint64) * (rng.random(K) < dens)).astype(np.uint32)
        got = g.device_alias(q)
        want = oracle_lib.alias(q)
        assert (got == want).all()
    got = g.device_alias(np.zeros(K, np.uint32))
    assert (got == oracle_lib.alias(np.zeros(K, np.uint32))).all()


def test_init_counts_match_oracle(gpu_lib, oracle_lib):
    K, V = 10000, 5
    C = np.array([1, 10, 100, 1000, 10000], np.uint32) * K
    with g.Sampler(0.1, 0.01, K, C, buffer_size=16, max_D=4, seed=5, chain=2) as s:
        n = s.read_state(q=False, alias=False, A=False, S=False, nnz=False)["n"]
    want = oracle_lib.init_counts(K, C, 0.01, 5, 2)
    assert (n == want).all()
    n = n.reshape(V, K)
    for w, lam in enumerate([10, 100, 1000, 10000][0:], start=1):
        assert 0.9 * lam <= n[w].mean() <= 1.1 * lam and 0.9 * lam <= n[w].var() <= 1.1 * lam


def _compare_phi(st, phi):
    import oracle
    K = len(st["S"])
    st = dict(st, alias=oracle.live_alias_entries(st["alias"], st["nnz"], K))
    phi = dict(phi, alias=oracle.live_alias_entries(phi["alias"], phi["nnz"], K))
    for key in ("S", "q", "A", "nnz", "alias"):
        a, b = st[key], phi[key]
        if not (a == b).all():
            bad = np.nonzero(a != b)[0]
            raise AssertionError(f"{key} differs at {bad[:8]}: gpu {a[bad[:8]]} oracle {b[bad[:8]]}")


def test_small_chain_parity(gpu_lib, oracle_lib, small_corpus):
    """100 free-running iterations of the small workload through the reference
    protocol (one buffer per iteration), checked after every stage."""
    c = small_corpus
    z_gpu = c.z.copy()
    z_orc = c.z.copy()
    kd = c.k_d()
    with g.Sampler(c.alpha, c.beta, c.K, c.counts, buffer_size=c.n_tokens, max_D=c.n_docs, seed=11,
                   flags=g.GPULDA_FLAG_LOGLIK) as s:
        ch = oracle_lib.Chain(c.K, c.alpha, c.beta, c.counts, seed=11)
        assert (s.read_state(q=False, alias=False, A=False, S=False, nnz=False)["n"] == ch.n).all()
        for it in range(100):
            s.sample_phi()
            ch.sample_phi()
            _compare_phi(s.read_state(n=False), ch.phi)
            s.sweep_buffer(0, z_gpu, c.w, c.d_len, kd)
            r = ch.sweep(c.w, z_orc, c.d_len, want_ll=True)
            assert (z_gpu == z_orc).all(), f"iteration {it}: {(z_gpu != z_orc).sum()} topics differ"
            n = s.read_state(q=False, alias=False, A=False, S=False, nnz=False)["n"]
            assert (n == ch.n).all(), f"iteration {it}: counts differ"
            ll, skipped = s.loglik()
            assert abs(ll - r["ll"]) <= LL_RTOL * abs(r["ll"]), (it, ll, r["ll"])
            assert skipped == r["ll_skipped"]
            cnt = s.counters()
            assert cnt["tokens"] == c.n_tokens and cnt["docs"] == c.n_docs
            assert cnt["sparse_work"] == int(r["stats"][2]) and cnt["sparse_draws"] == int(r["stats"][3])
    # the chain mixed: log-likelihood per token improved
    assert (z_gpu != c.z).mean() > 0.5


def test_small_chain_golden(gpu_lib, small_corpus):
    """Five iterations of the small workload through the reference protocol
    against the committed golden fixture (digests of the oracle's topics and
    counts after every iteration): no oracle runs beside it."""
    import hashlib
    import json
    import os
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "golden", "small_chain.json")) as f:
        golden = json.load(f)
    c = small_corpus
    z = c.z.astype(np.uint32).copy()
    sha = lambda a: hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()
    with g.Sampler(c.alpha, c.beta, c.K, c.counts, buffer_size=c.n_tokens, max_D=c.n_docs,
                   seed=golden["sampler_seed"], flags=g.GPULDA_FLAG_LOGLIK) as s:
        for w in golden["iterations"]:
            s.sample_phi()
            s.sweep_buffer(0, z, c.w, c.d_len, c.k_d())
            n = s.read_state(q=False, alias=False, A=False, S=False, nnz=False)["n"]
            assert z[:64].tolist() == w["z_first_64"], w["t"]
            assert sha(z) == w["sha256_z"], w["t"]
            assert sha(n.astype(np.uint32)) == w["sha256_n"], w["t"]
            ll, skipped = s.loglik()
            assert abs(ll - w["ll"]) <= LL_RTOL * abs(w["ll"]) and skipped == w["ll_skipped"], (w["t"], ll)
            cnt = s.counters()
            assert cnt["sparse_work"] == w["sparse_work"] and cnt["sparse_draws"] == w["sparse_draws"], w["t"]


def test_buffers_and_corpus_mode_agree(gpu_lib, oracle_lib, small_corpus):
    """Splitting the corpus into buffers (max_D = 300 documents, as the
    reference's fill_buffer does) or keeping it resident gives the same chain."""
    c = small_corpus
    iters = 3
    # resident corpus
    with g.Sampler(c.alpha, c.beta, c.K, c.counts, buffer_size=16, max_D=4, seed=3) as s:
        s.corpus_load(c.z.copy(), c.w, c.d_len)
        s.corpus_sweep(iters)
        z_res = s.corpus_z()
    # many buffers, reference protocol
    from gpupolyaurnlda_b200.train import iterate_buffers
    z_buf = c.z.copy()
    with g.Sampler(c.alpha, c.beta, c.K, c.counts, buffer_size=40000, max_D=300, seed=3) as s:
        for _ in range(iters):
            s.sample_phi()
            for z, w, d, kd in iterate_buffers(z_buf, c.w, c.d_len, c.k_d(), 40000, 300):
                s.sweep_buffer(0, z, w, d, kd)
    ch = oracle_lib.Chain(c.K, c.alpha, c.beta, c.counts, seed=3)
    z_orc = c.z.copy()
    for _ in range(iters):
        ch.sample_phi()
        ch.sweep(c.w, z_orc, c.d_len)
    assert (z_res == z_orc).all()
    assert (z_buf == z_orc).all()


def test_buffer_lengths_rewritten_in_place(gpu_lib, oracle_lib, small_corpus):
    """The host-buffer sweep reuses its pieces and document order while the
    lengths array is unchanged; rewriting the same arrays in place between
    iterations (documents in reverse order: same counts and totals) must be
    noticed, and the chain must still equal the oracle's."""
    c = small_corpus
    d = c.d_len.astype(np.uint32).copy()
    w = c.w.astype(np.uint32).copy()
    kd = c.k_d().astype(np.uint32).copy()
    z_gpu = c.z.astype(np.uint32).copy()
    z_orc = z_gpu.copy()
    ch = oracle_lib.Chain(c.K, c.alpha, c.beta, c.counts, seed=5)
    with g.Sampler(c.alpha, c.beta, c.K, c.counts, buffer_size=c.n_tokens, max_D=c.n_docs, seed=5) as s:
        for it in range(5):
            if it in (2, 4):
                offs = np.concatenate([[0], np.cumsum(d.astype(np.int64))])
                perm = np.concatenate([np.arange(offs[i], offs[i + 1]) for i in range(len(d) - 1, -1, -1)])
                d[:] = d[::-1].copy()
                kd[:] = kd[::-1].copy()
                w[:] = w[perm]
                z_gpu[:] = z_gpu[perm]
                z_orc[:] = z_orc[perm]
            s.sample_phi()
            ch.sample_phi()
            s.sweep_buffer(0, z_gpu, w, d, kd)
            ch.sweep(w, z_orc, d)
            assert (z_gpu == z_orc).all(), f"iteration {it}: {(z_gpu != z_orc).sum()} topics differ"


def test_sample_topics_concentrated(gpu_lib):
    """src/cu/test/test_topics.cu:276-334 restated: Phi concentrated on topic 0
    (beta = 0, counts only in topic 0) sends every token to topic 0."""
    K, V = 5, 3
    with g.Sampler(0.1, 0.0, K, np.ones(V, np.uint32), buffer_size=5, max_D=2) as s:
        n = np.zeros(V * K, np.uint32)
        n[0::K] = 50
        s.write_counts(n)
        s.sample_phi()
        st = s.read_state()
        assert (st["q"].reshape(V, K)[:, 1:] == 0).all()
        z = np.array([4, 1, 0, 4, 0], np.uint32)
        s.sweep_buffer(0, z, np.zeros(5, np.uint32), np.array([3, 2], np.uint32), np.array([1, 1], np.uint32))
        assert (z == 0).all()
        n = s.read_state()["n"]
        assert n[0] == 5 and n.sum() == 5


def test_edge_cases(gpu_lib, oracle_lib):
    K, V = 7, 11
    counts = np.arange(V, 0, -1).astype(np.uint32)
    with g.Sampler(0.5, 0.1, K, counts, buffer_size=64, max_D=8, seed=9) as s:
        s.sample_phi()
        phi = s.read_state(n=False)
        # empty buffer: no work, no error
        s.sweep_buffer(0, np.zeros(0, np.uint32), np.zeros(0, np.uint32), np.zeros(0, np.uint32))
        # ragged documents, including empty ones and single tokens; exactly buffer_size tokens
        d = np.array([0, 1, 30, 0, 1, 20, 12, 0], np.uint32)
        rng = np.random.default_rng(2)
        w = rng.integers(0, V, 64).astype(np.uint32)
        z = rng.integers(0, K, 64).astype(np.uint32)
        z_orc = z.copy()
        s.sweep_buffer(0, z, w, d)
        r = oracle_lib.z_sweep(K, V, 0.5, phi, w, z_orc, d, 0, key0=9)
        assert (z == z_orc).all()
        # too many tokens / documents: rejected before any work
        with pytest.raises(g.GpuldaError) as e:
            s.sweep_buffer(0, np.zeros(65, np.uint32), np.zeros(65, np.uint32), np.array([65], np.uint32))
        assert e.value.code == g.GPULDA_ERR_BUFFER
        with pytest.raises(g.GpuldaError) as e:
            s.sweep_buffer(0, np.zeros(9, np.uint32), np.zeros(9, np.uint32), np.ones(9, np.uint32))
        assert e.value.code == g.GPULDA_ERR_BUFFER
        # a topic id >= K is reported by the device, not written out of bounds
        zb = np.full(4, K + 3, np.uint32)
        with pytest.raises(g.GpuldaError) as e:
            s.sweep_buffer(0, zb, np.zeros(4, np.uint32), np.array([4], np.uint32))
        assert e.value.code == g.GPULDA_ERR_DEVICE
    # K = 1: every token stays in topic 0
    with g.Sampler(0.1, 0.01, 1, counts, buffer_size=64, max_D=8) as s:
        s.sample_phi()
        z = np.zeros(10, np.uint32)
        s.sweep_buffer(0, z, np.arange(10, dtype=np.uint32), np.array([10], np.uint32))
        assert (z == 0).all()


def test_protocol_errors(gpu_lib):
    L = g.lib()
    L.gpulda_set_fatal_errors(0)
    L.sample_phi()
    assert L.gpulda_last_error() == g.GPULDA_ERR_STATE
    args = g.make_args(0.1, 0.01, 40000, np.ones(3, np.uint32), 8, 2)
    bufs = (g.Buffer * 1)()
    assert L.gpulda_initialize_ex(args, bufs, 1, None) == g.GPULDA_ERR_UNSUPPORTED


@pytest.mark.parametrize("K", [1000, 16384])
def test_mid_slice_teacher_forced(gpu_lib, oracle_lib, K):
    """One iteration of a slice of the mid workload (K=1000, and a K above the
    shared-memory alias limit), teacher-forced: the oracle starts from the
    GPU's counts."""
    from gpupolyaurnlda_b200 import corpus
    import dataclasses
    wl = dataclasses.replace(corpus.WORKLOADS["mid"], K=K, V=20000 if K == 1000 else 3000,
                             D=20000 if K == 1000 else 2000)
    c = corpus.generate(wl, seed=4, device="cuda")
    with g.Sampler(c.alpha, c.beta, c.K, c.counts, buffer_size=c.n_tokens, max_D=c.n_docs, seed=1) as s:
        z_gpu = c.z.copy()
        for it in range(2):
            n_prev = s.read_state(q=False, alias=False, A=False, S=False, nnz=False)["n"]
            s.sample_phi()
            phi = oracle_lib.phi_step(c.K, c.V, c.beta, n_prev, it, 1, 0)
            _compare_phi(s.read_state(n=False), phi)
            z_orc = z_gpu.copy()
            s.sweep_buffer(0, z_gpu, c.w, c.d_len)
            r = oracle_lib.z_sweep(c.K, c.V, c.alpha, phi, c.w, z_orc, c.d_len, it, key0=1)
            assert (z_gpu == z_orc).all()
            n = s.read_state(q=False, alias=False, A=False, S=False, nnz=False)["n"]
            assert (n == r["n"]).all()
            # size-independent properties
            assert int(n.sum()) == c.n_tokens
            assert (np.bincount(c.w.astype(np.int64) * c.K + z_gpu, minlength=c.K * c.V) == n).all()


def test_count_rebuild_from_resident_topics(gpu_lib, oracle_lib, small_corpus):
    """gpulda_corpus_count_rebuild (warp-aggregated atomics) rebuilds exactly
    the counts the sweep rebuilt, n[w][z] = #tokens (reference: the per-token
    atomicAdd of src/cu/topics.cu:95), and resuming from them continues the
    same chain as the oracle."""
    c = small_corpus
    with g.Sampler(c.alpha, c.beta, c.K, c.counts, buffer_size=16, max_D=4, seed=4) as s:
        s.corpus_load(c.z.copy(), c.w, c.d_len)
        s.corpus_sweep(2)
        n_sweep = s.read_state(q=False, alias=False, A=False, S=False, nnz=False)["n"]
        z = s.corpus_z()
        ms = s.corpus_count_rebuild()
        assert ms > 0
        n_re = s.read_state(q=False, alias=False, A=False, S=False, nnz=False)["n"]
        assert (n_re == n_sweep).all()
        assert (n_re == np.bincount(c.w.astype(np.int64) * c.K + z, minlength=c.K * c.V)).all()
        s.corpus_sweep(1)
        z3 = s.corpus_z()
    ch = oracle_lib.Chain(c.K, c.alpha, c.beta, c.counts, seed=4)
    z_orc = c.z.copy()
    for _ in range(3):
        ch.sample_phi()
        ch.sweep(c.w, z_orc, c.d_len)
    assert (z3 == z_orc).all()
