"""Batched chains (include/gpulda_batch.h) against the CPU oracle and solo
runs: every problem of a batch -- K buckets of 64, 256, 1024 and 2048 topics
side by side, two problems sharing a bucket -- must give the topics and counts
of the oracle's chain (and of its solo Sampler run) with the same seed and
chain bit for bit, and the same joint log-likelihood within 1e-4 relative,
through graph replays, a change of launch shapes, and an autotuning pass
(which must leave the chains untouched)."""
import dataclasses
import json

import numpy as np
import pytest

import gpupolyaurnlda_b200 as g
from gpupolyaurnlda_b200 import corpus
from gpupolyaurnlda_b200.batch import (BATCH_MERGED, BATCH_MERGED_SWEEP, BATCH_PER_BUCKET, BatchChains,
                                       ProblemSpec)

pytestmark = pytest.mark.gpu

# (K, V, D, seed, chain): two K=50 problems share the first bucket
_PROBLEMS = [(50, 800, 300, 11, 0), (1000, 3000, 400, 12, 3), (20, 500, 200, 13, 1), (200, 2000, 350, 14, 0),
             (2048, 1500, 120, 15, 7), (50, 600, 250, 16, 2)]


def _specs():
    out = []
    for K, V, D, seed, chain in _PROBLEMS:
        wl = corpus.Workload(f"b{K}", K, V, D, 50.0 / K, 0.01, ("lognormal", 4.5, 1.0, 1, 3000), 1.05)
        c = corpus.generate(wl, seed=seed)
        out.append(ProblemSpec(c.alpha, c.beta, K, c.counts, c.z, c.w, c.d_len, seed=seed, chain=chain))
    return out


def _solo(spec, n_iter):
    """Topics, counts and per-iteration log-likelihoods of the solo chain."""
    lls = []
    with g.Sampler(spec.alpha, spec.beta, spec.K, spec.counts, buffer_size=16, max_D=4, seed=spec.seed,
                   chain=spec.chain, flags=g.GPULDA_FLAG_LOGLIK) as s:
        n0 = s.read_state(q=False, alias=False, A=False, S=False, nnz=False)["n"]
        s.corpus_load(spec.z.copy(), spec.w, spec.d_len)
        for _ in range(n_iter):
            s.corpus_sweep(1)
            lls.append(s.loglik()[0])
        z = s.corpus_z()
        n = s.read_state(q=False, alias=False, A=False, S=False, nnz=False)["n"]
    return z, n, lls, n0


@pytest.fixture(scope="module")
def specs(gpu_lib):
    return _specs()


@pytest.fixture(scope="module")
def solo(specs):
    return [_solo(s, 4) for s in specs]


def _check(b, specs, solo, it_ll):
    ll, _ = b.loglik()
    for p, s in enumerate(specs):
        z_s, n_s, lls, _ = solo[p]
        assert (b.z(p) == z_s).all(), f"problem {p}: topics differ"
        assert (b.counts(p) == n_s.reshape(-1)).all(), f"problem {p}: counts differ"
        assert abs(ll[p] - lls[it_ll]) <= 1e-4 * abs(lls[it_ll]), (p, ll[p], lls[it_ll])


def test_batch_equals_solo(specs, solo):
    with BatchChains(specs) as b:
        info = b.info()
        assert info["problems"] == len(specs) and info["buckets"] == 4
        assert info["tokens"] == sum(len(s.z) for s in specs)
        for p in range(len(specs)):  # initial counts
            assert (b.counts(p) == solo[p][3].reshape(-1)).all(), f"problem {p}: initial counts differ"
        b.sweep(1)
        ll1, _ = b.loglik()
        b.sweep(3)  # graph replays
        _check(b, specs, solo, 3)
    for p in range(len(specs)):
        assert abs(ll1[p] - solo[p][2][0]) <= 1e-4 * abs(solo[p][2][0])


def test_batch_equals_oracle_chains(specs, oracle_lib):
    """Each problem's chain in the batch against oracle.Chain directly: the
    initial counts, then topics, counts and log-likelihood after each of
    three iterations (reference semantics src/cu/polyaurn.cu:61-123,
    src/cu/topics.cu:36-105)."""
    chains = [oracle_lib.Chain(sp.K, sp.alpha, sp.beta, sp.counts, seed=sp.seed, chain=sp.chain) for sp in specs]
    zs = [sp.z.copy() for sp in specs]
    with BatchChains(specs) as b:
        for p, ch in enumerate(chains):
            assert (b.counts(p) == ch.n).all(), f"problem {p}: initial counts differ from the oracle"
        for it in range(3):
            b.sweep(1)
            ll, _ = b.loglik()
            for p, (sp, ch) in enumerate(zip(specs, chains)):
                ch.sample_phi()
                r = ch.sweep(sp.w, zs[p], sp.d_len, want_ll=True)
                assert (b.z(p) == zs[p]).all(), f"iteration {it}, problem {p}: topics differ from the oracle"
                assert (b.counts(p) == ch.n).all(), f"iteration {it}, problem {p}: counts differ from the oracle"
                assert abs(ll[p] - r["ll"]) <= 1e-4 * abs(r["ll"]), (it, p, ll[p], r["ll"])


def test_batch_shapes_and_autotuner_leave_chains_unchanged(specs, solo, tmp_path):
    cache = tmp_path / "tune.json"
    with BatchChains(specs) as b:
        assert b.info()["mode"] == BATCH_MERGED_SWEEP  # the default
        b.sweep(1)
        n_tuned = b.tune(str(cache))
        assert n_tuned == 5  # four buckets and the merged launches
        entries = json.loads(cache.read_text())
        bucket_keys = [k for k in entries if "|K<=" in k]
        merged_keys = [k for k in entries if "|merged|" in k]
        assert len(bucket_keys) == 4 and all(len(entries[k]) == 3 for k in bucket_keys)
        assert len(merged_keys) == 1 and len(entries[merged_keys[0]]) == 4
        assert entries[merged_keys[0]][3] in (BATCH_PER_BUCKET, BATCH_MERGED, BATCH_MERGED_SWEEP)
        # every mode, with other shapes: the chains must not change
        b.set_shapes([(2, 0, 4096), (4, 4, 16384), (8, 2, 100000), (2, 0, 7)])
        b.set_mode(BATCH_PER_BUCKET)
        assert b.info()["mode"] == BATCH_PER_BUCKET
        b.sweep(1)
        b.set_mode(BATCH_MERGED, (4, 2, 50000))
        b.sweep(1)
        b.set_mode(BATCH_MERGED_SWEEP, (2, 0, 65536))
        b.sweep(1)
        _check(b, specs, solo, 3)
    with BatchChains(specs) as b:
        assert b.tune(str(cache)) == 0  # every entry from the cache
        assert [list(s) for s in b.shapes()] == [entries[k] for k in sorted(bucket_keys,
                                                                           key=lambda k: int(k.split("<=")[1]))]
        assert b.info()["mode"] == entries[merged_keys[0]][3]


def test_batch_async_on_caller_stream(specs, solo):
    import torch
    st = torch.cuda.Stream()
    with BatchChains(specs) as b:
        b.sweep_async(4, st.cuda_stream)
        b.sync()
        _check(b, specs, solo, 3)
