"""Host-side pieces of the serving measurement on the CPU: requests drawn from
a model's own topics, the document-completion split, and the held-out
log-likelihood against a direct evaluation."""
import numpy as np

from gpupolyaurnlda_b200.serve import completion_loglik, model_requests, split_halves


def _fixed_point_phi(K, V, seed):
    rng = np.random.default_rng(seed)
    x = rng.integers(0, 5, (V, K)).astype(np.float64)
    x[:, 3] = 0
    x[7, 3] = 10  # a topic with one word
    S = x.sum(axis=0)
    q = np.floor(x * 2.0 ** 32 / np.where(S > 0, S, 1)).clip(0, 2 ** 32 - 1).astype(np.uint32)
    return q.reshape(-1)


def test_model_requests_follow_the_topics():
    K, V = 8, 50
    q = _fixed_point_phi(K, V, 1)
    lengths, words = model_requests(q, K, 300, seed=2, lo=1, hi=40, mu=2.5, device="cpu")
    assert lengths.dtype == np.uint32 and words.dtype == np.uint32
    assert words.size == lengths.sum() and lengths.min() >= 1 and lengths.max() <= 40
    assert words.max() < V
    # word 7 is topic 3's only word: it must appear (topic 3 gets tokens) and
    # every word drawn must have q > 0 in some topic
    assert (q.reshape(V, K)[words].max(axis=1) > 0).all()
    again = model_requests(q, K, 300, seed=2, lo=1, hi=40, mu=2.5, device="cpu")
    assert (again[0] == lengths).all() and (again[1] == words).all()  # seeded


def test_split_halves_and_completion_loglik():
    K, V = 8, 50
    q = _fixed_point_phi(K, V, 3)
    lengths, words = model_requests(q, K, 120, seed=4, lo=1, hi=30, mu=2.0, device="cpu")
    fl, fw, sl, sw = split_halves(lengths, words)
    assert (fl + sl == lengths).all() and (fl == (lengths.astype(np.int64) + 1) // 2).all()
    offs = np.concatenate([[0], np.cumsum(lengths.astype(np.int64))])
    first = np.concatenate([words[offs[i]:offs[i] + fl[i]] for i in range(len(lengths))])
    second = np.concatenate([words[offs[i] + fl[i]:offs[i + 1]] for i in range(len(lengths))])
    assert (fw == first).all() and (sw == second).all()
    theta = np.random.default_rng(5).dirichlet(np.ones(K), len(lengths)).astype(np.float32)
    tot, n = completion_loglik(q, K, theta, sl, sw, device="cpu")
    phi = q.reshape(V, K).astype(np.float64) / 2.0 ** 32
    so = np.concatenate([[0], np.cumsum(sl.astype(np.int64))])
    want, cnt = 0.0, 0
    for d in range(len(sl)):
        p = (phi[sw[so[d]:so[d + 1]]] * theta[d].astype(np.float64)).sum(axis=1)
        want += np.log(p[p > 0]).sum()
        cnt += int((p > 0).sum())
    assert n == cnt and abs(tot - want) <= 1e-9 * abs(want)
