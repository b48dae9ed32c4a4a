"""The committed golden fixture (tests/golden/small_chain.json, written by
tests/golden/make_golden.py): the synthetic small corpus and five iterations
of the CPU oracle's chain on it must reproduce it -- bit for bit for the
corpus, topics and counts; the log-likelihood within 1e-12 relative (the
oracle's threads sum it in their own order)."""
import json
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
import make_golden  # noqa: E402

with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "small_chain.json")) as f:
    GOLDEN = json.load(f)


def test_small_corpus_matches_golden(small_corpus):
    assert make_golden.corpus_digest(small_corpus) == GOLDEN["corpus"]


def test_oracle_chain_matches_golden(oracle_lib, small_corpus):
    got = make_golden.oracle_chain(small_corpus, len(GOLDEN["iterations"]))
    for g, w in zip(got, GOLDEN["iterations"]):
        for key in ("sha256_z", "sha256_n", "ll_skipped", "sparse_work", "sparse_draws", "z_first_64"):
            assert g[key] == w[key], (w["t"], key)
        assert abs(g["ll"] - w["ll"]) <= 1e-12 * abs(w["ll"]), (w["t"], g["ll"], w["ll"])
