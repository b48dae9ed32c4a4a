"""The CPU oracle against known answers.

* Published Philox4x32-10 known-answer vectors (Random123 distribution,
  Salmon et al. SC'11).
* The reference's own unit-test vectors for this path, restated for this
  design's integer formulation:
    src/cu/test/test_spalias.cu:14-53     build_alias, p = {.9, .02, .01 x 8}
    src/cu/test/test_topics.cu:16-47      compute_d_idx, lengths 1..n, n = 527
    src/cu/test/test_topics.cu:49-76      draw_alias, K=5, prob .5, alias 1
    src/cu/test/test_topics.cu:78-132     draw_wary_search, 96 slots
    src/cu/test/test_topics.cu:134-189    count_topics, z = i mod 25
    src/cu/test/test_topics.cu:191-237    compute_product_cumsum, m=i, Phi=6i
    src/cu/test/test_hashmap.cu:224-266   90 inserts of i mod 9 -> counts 10
    src/cu/test/test_polyaurn.cu:16-74    init mean/variance bands
    src/cu/test/test_polyaurn.cu:76-118   Phi ~ {.01,.09,.9} and {1/3,1/3,1/3}
    src/cu/test/test_polyaurn.cu:120-273  transpose / colsums (word-major
                                          layout, per-word sums)
    src/cu/test/test_topics.cu:276-334    sample_topics with Phi concentrated on
                                          topic 0 -> every z = 0
"""
import math

import numpy as np
import pytest

TWO32 = 4294967296


def test_philox_published_vectors(oracle_lib):
    ctr = np.array([[0, 0, 0, 0], [0xffffffff] * 4, [0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344]], np.uint32)
    keys = [(0, 0), (0xffffffff, 0xffffffff), (0xa4093822, 0x299f31d0)]
    want = [[0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8],
            [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd],
            [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]]
    for c, (k0, k1), w in zip(ctr, keys, want):
        assert oracle_lib.philox(c, k0, k1)[0].tolist() == w


def test_det_log_accuracy(oracle_lib):
    rng = np.random.default_rng(0)
    xs = np.concatenate([rng.random(2000) * 10.0 ** rng.integers(-12, 12, 2000), [1.0, 2.0, 0.5, 1e-300, 1e300]])
    for x in xs:
        x = float(x)
        if x <= 0:
            continue
        assert abs(oracle_lib.det_log(x) - math.log(x)) <= 4e-16 * max(1.0, abs(math.log(x)))
    assert oracle_lib.det_log(0.0) == -math.inf


# --- src/cu/test/test_spalias.cu:14-53 ---------------------------------------
def _alias_distribution(table: np.ndarray, K: int | None = None) -> np.ndarray:
    """Topic distribution of a table (entry: threshold | own << 32 | alias << 48)."""
    n = len(table)
    K = K or n
    thr = (table & 0xffffffff).astype(np.float64)
    own = ((table >> 32) & 0xffff).astype(np.int64)
    ali = (table >> 48).astype(np.int64)
    keep = np.where(thr == 0xffffffff, 1.0, thr / TWO32)
    p = np.zeros(K)
    np.add.at(p, own, keep / n)
    np.add.at(p, ali, (1 - keep) / n)
    return p


def test_alias_reference_vector(oracle_lib):
    # p = {.9, .02, .01 x 8} as integer weights: the single heavy item (0) is
    # everyone's alias and keeps its own slot.
    q = np.array([90, 2] + [1] * 8, np.uint32)
    t = oracle_lib.alias(q)
    assert ((t >> 48) == 0).all()
    assert (((t >> 32) & 0xffff) == np.arange(10)).all()
    keep = (t & 0xffffffff)
    assert keep[0] == 0xffffffff
    assert keep[1] == int(0.2 * TWO32) and (keep[2:] == int(0.1 * TWO32)).all()
    assert np.allclose(_alias_distribution(t), q / q.sum(), atol=1e-9)


def test_alias_distribution_random(oracle_lib):
    rng = np.random.default_rng(3)
    for K in (1, 2, 5, 20, 257, 1000):
        for dens in (1.0, 0.3, 0.02):
            q = (rng.integers(0, 2 ** 32, K, dtype=np.uint64) * (rng.random(K) < dens)).astype(np.uint32)
            if q.sum() == 0:
                q[K // 2] = 7
            t = oracle_lib.alias(q)
            p = _alias_distribution(t)
            assert np.allclose(p, q / q.astype(np.float64).sum(), atol=K * 2.0 ** -31)
            # zero-weight topics are never returned
            ali = (t >> 48).astype(np.int64)
            keep = t & 0xffffffff
            assert (q[ali[keep != 0xffffffff]] > 0).all()
            # the sparse form over the nonzero items gives the same distribution
            nzk = np.nonzero(q)[0]
            ts = oracle_lib.alias_items(q[nzk], nzk.astype(np.uint16))
            assert np.allclose(_alias_distribution(ts, K), q / q.astype(np.float64).sum(), atol=K * 2.0 ** -31)


# --- src/cu/test/test_topics.cu:16-47 ----------------------------------------
def test_doc_offsets_reference_vector(oracle_lib):
    n_docs = 2 * 256 + 15
    d_len = np.arange(1, 4 * 256 + 1, dtype=np.uint32)[:n_docs]
    idx = oracle_lib.doc_offsets(d_len)
    assert idx[0] == 0
    assert (idx[1:] == np.cumsum(d_len.astype(np.uint64))[:-1]).all()


# --- src/cu/test/test_topics.cu:49-76 ----------------------------------------
def test_alias_draw_reference_vector(oracle_lib):
    K = 5
    table = np.array([(1 << 48) | (s << 32) | (TWO32 // 2) for s in range(K)], np.uint64)
    # The reference draws with u = 0.6f (slot 3, remainder ~0 < .5 -> 3) and
    # u = 0.75f (slot 3, remainder .75 >= .5 -> alias 1); the slot word here is
    # u * 2^32 and the keep word is the remainder * 2^32.
    u6 = int(float(np.float32(0.6)) * TWO32)
    assert oracle_lib.alias_draw(table, u6, (u6 * K) % TWO32) == 3
    u75 = int(0.75 * TWO32)
    assert oracle_lib.alias_draw(table, u75, (u75 * K) % TWO32) == 1


# --- src/cu/test/test_topics.cu:78-132 ---------------------------------------
@pytest.mark.parametrize("u,want", [(0.0, 0), (0.02, 1), (0.16, 15), (0.4, 38), (0.985, 94), (1.0, 95)])
def test_sparse_select_reference_vector(oracle_lib, u, want):
    mass = np.ones(96, np.uint64)
    r = min(int(u * TWO32), TWO32 - 1)
    i, _ = oracle_lib.sparse_select(mass, r)
    assert i == want


# --- src/cu/test/test_topics.cu:134-189 and test_hashmap.cu:224-266 -----------
def test_count_topics_reference_vectors(oracle_lib):
    z = (np.arange(100) % 25).astype(np.uint32)
    d, c = oracle_lib.count_topics(z, 25)
    assert d == 25 and (c == 4).all()
    z = (np.arange(90) % 9).astype(np.uint32)
    d, c = oracle_lib.count_topics(z, 100)
    assert d == 9 and (c[:9] == 10).all() and (c[9:] == 0).all()


# --- src/cu/test/test_topics.cu:191-237 --------------------------------------
def test_product_cumsum_reference_vector(oracle_lib):
    i = np.arange(100, dtype=np.uint64)
    mass = i * (6 * i)  # m_k = k, Phi_k = 6k
    _, prefix = oracle_lib.sparse_select(mass, 0)
    excl = np.concatenate([[0], prefix[:-1]])
    im1 = i.astype(np.int64) - 1
    want = np.where(i == 0, 0, im1 * (im1 + 1) * (2 * im1 + 1))
    assert (excl.astype(np.int64) == want).all()
    assert int(prefix[-1]) == 99 * 100 * 199


# --- src/cu/test/test_polyaurn.cu:16-74 --------------------------------------
def test_init_counts_reference_bands(oracle_lib):
    K, V = 10000, 5
    C = np.array([1, 10, 100, 1000, 10000], np.uint32) * K
    n = oracle_lib.init_counts(K, C, 0.01).reshape(V, K)  # word-major
    for w, lam in enumerate([1, 10, 100, 1000, 10000]):
        m, v = n[w].mean(), n[w].var()
        if lam == 1:
            assert m <= 2 and v <= 2
        else:
            assert 0.9 * lam <= m <= 1.1 * lam and 0.9 * lam <= v <= 1.1 * lam


# --- src/cu/test/test_polyaurn.cu:76-273 -------------------------------------
def test_phi_step_reference_rows(oracle_lib):
    K = V = 3
    # reference layout is topic-major n[k][v]; this library is word-major n[v][k]
    n_topic_major = np.array([[1, 10, 100], [1, 1, 1], [1000, 1000, 1000]], np.uint32)
    n = np.ascontiguousarray(n_topic_major.T).reshape(-1)
    acc = np.zeros((3, 3))
    hits = np.zeros(3)
    reps = 2000  # the {1,1,1} row's per-draw spread is ~0.3: the mean needs many draws
    for t in range(reps):
        phi = oracle_lib.phi_step(K, V, 0.01, n, t, threads=1)
        q = phi["q"].reshape(V, K).astype(np.float64) / TWO32
        live = phi["S"] > 0  # a topic whose draws are all zero has Phi = 0
        acc[live] += q.T[live]
        hits += live
        # word-major layout and per-word sums (transpose + colsums tests)
        assert (phi["A"] == phi["q"].reshape(V, K).astype(np.uint64).sum(1)).all()
        assert np.allclose(q.sum(0), live.astype(np.float64), atol=1e-8)  # each live topic's Phi sums to 1
    mean = acc / hits[:, None]
    assert np.allclose(mean[0], [0.01, 0.09, 0.9], atol=0.02)
    assert np.allclose(mean[1], [1 / 3] * 3, atol=0.02)
    assert np.allclose(mean[2], [1 / 3] * 3, atol=0.02)


def test_phi_step_matches_direct_computation(oracle_lib):
    rng = np.random.default_rng(5)
    K, V, beta, t = 7, 11, 0.05, 3
    n = rng.integers(0, 200, K * V).astype(np.uint32)
    n[::5] = 0
    phi = oracle_lib.phi_step(K, V, beta, n, t, 9, 4)
    x = oracle_lib.poisson(n, np.arange(K * V, dtype=np.uint64), beta, t, oracle_lib.STREAM_PHI, 9, 4)
    S = x.reshape(V, K).astype(np.uint64).sum(0)
    assert (phi["S"] == S).all()
    q = np.zeros(K * V, np.uint64)
    for c in range(K * V):
        if x[c]:
            q[c] = min((int(x[c]) << 32) // int(S[c % K]), 0xffffffff)
    assert (phi["q"] == q).all()
    assert (phi["nnz"] == (x.reshape(V, K) > 0).sum(1)).all()
    for w in range(V):
        row = phi["q"][w * K:(w + 1) * K]
        nzk = np.nonzero(row)[0]
        assert phi["nnz"][w] == len(nzk)
        assert (phi["alias"][w * K:w * K + len(nzk)] == oracle_lib.alias_items(row[nzk], nzk.astype(np.uint16))).all()


# --- src/cu/test/test_topics.cu:276-334 --------------------------------------
def test_sample_topics_concentrated(oracle_lib):
    K, V = 5, 3
    # beta = 0 and counts only in topic 0 -> x (hence Phi) is zero elsewhere
    n = np.zeros(V * K, np.uint32)
    n[0::K] = 50
    phi = oracle_lib.phi_step(K, V, 0.0, n, 0)
    assert (phi["q"].reshape(V, K)[:, 1:] == 0).all()
    z = np.array([4, 1, 0, 4, 0], np.uint32)
    w = np.zeros(5, np.uint32)
    d = np.array([3, 2], np.uint32)
    r = oracle_lib.z_sweep(K, V, 0.1, phi, w, z, d, 0)
    assert (z == 0).all()
    assert r["n"][0] == 5 and r["n"].sum() == 5
