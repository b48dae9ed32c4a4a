"""Fold-in serving (include/gpulda_serve.h) against the CPU oracle: theta bit
for bit and the per-request log-likelihood within 1e-9 relative, for a model
copied from a trained single model and for one built from its fixed-point
Phi; each request's result is the same alone, in a mix of many, one launch per
document, and under a request pool so small that admissions must wait."""
import dataclasses

import numpy as np
import pytest

import gpupolyaurnlda_b200 as g
from gpupolyaurnlda_b200 import corpus
from gpupolyaurnlda_b200.serve import Server, zipf_requests

pytestmark = pytest.mark.gpu

N_ITER = 6


@pytest.fixture(scope="module")
def model(gpu_lib):
    """A K=200 model after three training iterations, its state on the host,
    and a serving handle copied from it."""
    wl = corpus.Workload("serve", 200, 3000, 400, 0.25, 0.01, ("lognormal", 4.5, 0.8, 5, 2000), 1.05)
    c = corpus.generate(wl, seed=21)
    s = g.Sampler(c.alpha, c.beta, c.K, c.counts, buffer_size=16, max_D=4, seed=4)
    s.corpus_load(c.z.copy(), c.w, c.d_len)
    s.corpus_sweep(3)
    st = s.read_state(n=False, S=False)
    srv = Server(N_ITER, slots=4, seed=9, chain=2)  # persistent, 4 request warps per SM
    s.close()  # the server holds its own copy
    yield c, st, srv
    srv.close()


def _requests(V, n, seed):
    lengths, words = zipf_requests(n, V, seed, mu=4.0, sigma=1.2, lo=1, hi=3000)
    lengths[:3] = [0, 1, 3000]  # empty, single token, longest
    words = np.resize(words, int(lengths.sum())).astype(np.uint32)
    return lengths, words


def _run(srv, ids, lengths, words, chunk=None):
    chunk = chunk or len(ids)
    offs = np.concatenate([[0], np.cumsum(lengths.astype(np.int64))])
    for a in range(0, len(ids), chunk):
        b = min(len(ids), a + chunk)
        srv.submit(ids[a:b], lengths[a:b], words[offs[a]:offs[b]])
        srv.progress()
    srv.drain()
    out = srv.poll(len(ids) + 8)
    assert len(out["ids"]) == len(ids)
    order = np.argsort(out["ids"])
    pos = np.searchsorted(out["ids"][order], ids)
    return {k: (v[order][pos] if v is not None else None) for k, v in out.items()}


def test_fold_in_matches_oracle(model, oracle_lib):
    c, st, srv = model
    lengths, words = _requests(c.V, 60, 5)
    ids = np.arange(1000, 1060, dtype=np.uint64) | (np.uint64(7) << np.uint64(40))  # high id bits in use
    got = _run(srv, ids, lengths, words)
    ref = oracle_lib.fold_in(c.K, c.V, c.alpha, st, words, lengths, ids, N_ITER, seed=9, chain=2)
    assert (got["theta"].view(np.uint32) == ref["theta"].view(np.uint32)).all()
    assert (got["skipped"] == ref["skipped"]).all()
    np.testing.assert_allclose(got["ll"], ref["ll"], rtol=1e-9, atol=1e-9)
    assert np.allclose(got["theta"].sum(axis=1), 1.0, atol=1e-4)


def test_same_alone_mixed_unbatched_and_memory_bound(model):
    c, st, srv = model
    lengths, words = _requests(c.V, 300, 6)
    ids = np.arange(300, dtype=np.uint64) * np.uint64(2654435761)
    mixed = _run(srv, ids, lengths, words, chunk=37)
    offs = np.concatenate([[0], np.cumsum(lengths.astype(np.int64))])
    for r in (0, 2, 17, 299):  # alone
        one = _run(srv, ids[r:r + 1], lengths[r:r + 1], words[offs[r]:offs[r + 1]])
        assert (one["theta"][0].view(np.uint32) == mixed["theta"][r].view(np.uint32)).all()
        assert one["ll"][0] == mixed["ll"][r]
    # one launch per document, and a pool that holds only a few requests
    q = st["q"]
    for kw in (dict(mode="launch", max_batch=1, slots=16), dict(mode="launch", max_batch=40, slots=3),
               dict(slots=1, pool_bytes=28_000), dict(mode="launch", slots=2, pool_bytes=28_000),
               dict(max_inflight=5)):
        with Server(N_ITER, seed=9, chain=2, q=q, K=c.K, alpha=c.alpha, **kw) as s2:
            other = _run(s2, ids, lengths, words, chunk=50)
            stats = s2.stats()
            assert (other["theta"].view(np.uint32) == mixed["theta"].view(np.uint32)).all()
            assert (other["ll"] == mixed["ll"]).all()
            assert stats["pool_used"] == 0 and stats["inflight"] == 0
            if kw.get("max_batch") == 1:
                assert stats["launches"] == len(ids)
            if "pool_bytes" in kw or "max_inflight" in kw:
                assert stats["deferred"] > 0


def test_model_from_phi_equals_copied_model(model):
    c, st, srv = model
    with Server(N_ITER, seed=9, chain=2, q=st["q"], K=c.K, alpha=c.alpha) as s2:
        lengths, words = _requests(c.V, 40, 8)
        ids = np.arange(40, dtype=np.uint64)
        a = _run(srv, ids, lengths, words)
        b = _run(s2, ids, lengths, words)
        assert (a["theta"].view(np.uint32) == b["theta"].view(np.uint32)).all()


def test_submit_rejects_bad_requests(model):
    c, st, srv = model
    with pytest.raises(g.GpuldaError) as e:
        srv.submit([1], [2], np.array([0, c.V], np.uint32))
    assert e.value.code == 2
    with pytest.raises(g.GpuldaError) as e:
        srv.submit([1], [70000], np.zeros(70000, np.uint32))
    assert e.value.code == 7
    with Server(N_ITER, q=st["q"], K=c.K, alpha=c.alpha, pool_bytes=4096) as s2:
        with pytest.raises(g.GpuldaError) as e:
            s2.submit([1], [2000], np.zeros(2000, np.uint32))
        assert e.value.code == 7
    assert srv.stats()["queued"] == 0
