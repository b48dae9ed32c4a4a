"""Writes tests/golden/small_chain.json: digests of the small workload's
corpus and of five iterations of the CPU oracle's chain on it.

The fixture pins the synthetic-corpus generator and the oracle against drift
(tests/test_golden.py re-derives both on the CPU), and gives the GPU test a
committed answer that does not depend on running the oracle beside it
(tests/test_gpu_parity.py::test_small_chain_golden).  Regenerate only on a
deliberate change of the generator or of the sampler's definition:

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

SEED = 11          # sampler seed (Philox key word 0); chain 0
ITERATIONS = 5


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def corpus_digest(c) -> dict:
    return {"K": c.K, "V": c.V, "D": c.n_docs, "N": c.n_tokens, "alpha": c.alpha, "beta": c.beta,
            "sha256_w": sha(c.w.astype(np.uint32)), "sha256_z0": sha(c.z.astype(np.uint32)),
            "sha256_d_len": sha(c.d_len.astype(np.uint32)), "sha256_counts": sha(c.counts.astype(np.uint32))}


def oracle_chain(c, iterations: int = ITERATIONS) -> list[dict]:
    import oracle
    ch = oracle.Chain(c.K, c.alpha, c.beta, c.counts, seed=SEED)
    z = c.z.astype(np.uint32).copy()
    out = []
    for t in range(iterations):
        ch.sample_phi()
        r = ch.sweep(c.w, z, c.d_len, want_ll=True)
        out.append({"t": t, "sha256_z": sha(z), "sha256_n": sha(ch.n.astype(np.uint32)), "ll": float(r["ll"]),
                    "ll_skipped": int(r["ll_skipped"]), "sparse_work": int(r["stats"][2]),
                    "sparse_draws": int(r["stats"][3]), "z_first_64": z[:64].tolist()})
    return out


def main() -> None:
    from gpupolyaurnlda_b200 import corpus
    from oracle.build import build_oracle
    build_oracle()
    c = corpus.generate("small", seed=1)
    doc = {"workload": "small (seed 1)", "corpus": corpus_digest(c), "sampler_seed": SEED,
           "iterations": oracle_chain(c)}
    with open(os.path.join(HERE, "small_chain.json"), "w") as f:
        json.dump(doc, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
