"""Properties of the CPU oracle's sweep that do not depend on size.

* the conditional it samples from is p(z=k) ~ Phi[k][w] (alpha + m_dk^-i)
  (src/cu/topics.cu:59-98 structure), checked by a chi-square test;
* counts rebuilt by the sweep equal the histogram of the new topics;
* results do not depend on the thread count, on how the corpus is split into
  buffers (src/train.rs:86-97), or on stopping and resuming the chain.
"""
import numpy as np
import pytest

TWO32 = 4294967296


def _tiny_phi(oracle_lib, K=6, V=3, seed=0):
    rng = np.random.default_rng(seed)
    n = rng.integers(0, 30, K * V).astype(np.uint32)
    return oracle_lib.phi_step(K, V, 0.1, n, 0)


def test_single_token_conditional(oracle_lib):
    """A document of two tokens with z = (3, 4): the first token is resampled
    with the second's topic in m^-i, so over many iterations its topic
    follows q[w][k] (alpha + [k == 4])."""
    K, V, alpha = 6, 3, 0.3
    phi = _tiny_phi(oracle_lib, K, V)
    q = phi["q"].reshape(V, K).astype(np.float64)
    w = np.array([1, 2], np.uint32)
    T = 20000
    hits = np.zeros(K)
    for t in range(T):
        z = np.array([3, 4], np.uint32)
        oracle_lib.z_sweep(K, V, alpha, phi, w, z, np.array([2], np.uint32), t, threads=1)
        hits[z[0]] += 1
    # token 0: m^-i has only z_1 = 4
    p = q[1] * (alpha + (np.arange(K) == 4))
    p /= p.sum()
    expected = p * T
    mask = expected > 5
    chi2 = (((hits - expected) ** 2)[mask] / expected[mask]).sum()
    assert chi2 < 25.0, (hits, expected)


def test_counts_equal_histogram(oracle_lib, small_corpus):
    c = small_corpus
    ch = oracle_lib.Chain(c.K, c.alpha, c.beta, c.counts, seed=2)
    z = c.z.copy()
    ch.sample_phi()
    r = ch.sweep(c.w, z, c.d_len)
    hist = np.bincount(c.w.astype(np.int64) * c.K + z, minlength=c.K * c.V)
    assert (r["n"] == hist).all()
    assert int(r["stats"][0]) == c.n_tokens and int(r["stats"][1]) == c.n_docs


def test_thread_count_and_buffer_split_invariance(oracle_lib, small_corpus):
    c = small_corpus
    outs = []
    for threads, split in ((1, None), (8, None), (3, 700)):
        ch = oracle_lib.Chain(c.K, c.alpha, c.beta, c.counts, seed=4, threads=threads)
        z = c.z.copy()
        for _ in range(3):
            ch.sample_phi()
            if split is None:
                ch.sweep(c.w, z, c.d_len)
            else:
                t0 = int(c.d_len[:split].sum())
                za, zb = z[:t0].copy(), z[t0:].copy()
                ch.sweep(c.w[:t0], za, c.d_len[:split])
                ch.sweep(c.w[t0:], zb, c.d_len[split:])
                z = np.concatenate([za, zb])
        outs.append((z, ch.n.copy()))
    for z, n in outs[1:]:
        assert (z == outs[0][0]).all() and (n == outs[0][1]).all()


def test_resume_is_bit_identical(oracle_lib, small_corpus):
    """z is the whole Gibbs state (n is rebuilt from it); random streams are
    keyed by (seed, iteration, token), so stopping after iteration 2 and
    resuming from the saved z and counts reproduces the uninterrupted chain."""
    c = small_corpus
    ch = oracle_lib.Chain(c.K, c.alpha, c.beta, c.counts, seed=6)
    z = c.z.copy()
    for _ in range(5):
        ch.sample_phi()
        ch.sweep(c.w, z, c.d_len)
        if ch.t == 1:
            saved = (z.copy(), ch.n.copy(), ch.t)
    ch2 = oracle_lib.Chain(c.K, c.alpha, c.beta, c.counts, seed=6)
    z2, ch2.n, ch2.t = saved[0].copy(), saved[1].copy(), saved[2]
    for _ in range(3):
        ch2.sample_phi()
        ch2.sweep(c.w, z2, c.d_len)
    assert (z2 == z).all() and (ch2.n == ch.n).all()


def test_chains_differ_by_chain_id(oracle_lib, small_corpus):
    c = small_corpus
    zs = []
    for chain in (0, 1):
        ch = oracle_lib.Chain(c.K, c.alpha, c.beta, c.counts, seed=0, chain=chain)
        z = c.z.copy()
        ch.sample_phi()
        ch.sweep(c.w, z, c.d_len)
        zs.append(z)
    assert (zs[0] != zs[1]).mean() > 0.3


def test_loglik_improves(oracle_lib, small_corpus):
    c = small_corpus
    ch = oracle_lib.Chain(c.K, c.alpha, c.beta, c.counts, seed=0)
    z = c.z.copy()
    lls = []
    for _ in range(15):
        ch.sample_phi()
        lls.append(ch.sweep(c.w, z, c.d_len, want_ll=True)["ll"])
    assert lls[-1] > lls[0] + 0.1 * abs(lls[0])


def test_fold_in_properties(oracle_lib, small_corpus):
    """Fold-in of new documents against a fixed model (the serving path's
    definition): theta is a distribution with the (m + alpha) / (L + K alpha)
    form, a result depends only on its request id and words (not on the other
    requests of the call, their order or the thread count), and different ids
    draw differently."""
    c = small_corpus
    ch = oracle_lib.Chain(c.K, c.alpha, c.beta, c.counts, seed=2)
    ch.sample_phi()
    ch.sweep(c.w, c.z.astype(np.uint32).copy(), c.d_len)
    ch.sample_phi()
    phi = ch.phi
    rng = np.random.default_rng(0)
    lengths = rng.integers(5, 200, 12).astype(np.uint32)
    words = rng.integers(0, c.V, int(lengths.sum())).astype(np.uint32)
    ids = np.arange(100, 112, dtype=np.uint64)
    r = oracle_lib.fold_in(c.K, c.V, c.alpha, phi, words, lengths, ids, 20, seed=2)
    assert np.allclose(r["theta"].sum(axis=1), 1.0, atol=1e-5)
    m = np.rint((r["theta"].astype(np.float64) * (lengths[:, None] + c.K * c.alpha)) - c.alpha)
    assert (m.sum(axis=1) == lengths).all() and (m >= 0).all()
    assert np.isfinite(r["ll"]).all() and (r["ll"] < 0).all()
    # each request alone, in reverse order, and with one thread
    offs = np.concatenate([[0], np.cumsum(lengths.astype(np.int64))])
    for i in (0, 5, 11):
        one = oracle_lib.fold_in(c.K, c.V, c.alpha, phi, words[offs[i]:offs[i + 1]], lengths[i:i + 1], ids[i:i + 1],
                                 20, seed=2, threads=1)
        assert (one["theta"][0] == r["theta"][i]).all() and one["ll"][0] == r["ll"][i]
    rev = oracle_lib.fold_in(c.K, c.V, c.alpha, phi,
                             np.concatenate([words[offs[i]:offs[i + 1]] for i in range(11, -1, -1)]),
                             lengths[::-1].copy(), ids[::-1].copy(), 20, seed=2)
    assert (rev["theta"][::-1] == r["theta"]).all()
    other = oracle_lib.fold_in(c.K, c.V, c.alpha, phi, words, lengths, ids + np.uint64(1000), 20, seed=2)
    assert (other["theta"] != r["theta"]).any()
