import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: longer CPU test")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle.build import build_oracle
    build_oracle()
    import oracle
    return oracle


@pytest.fixture(scope="session")
def small_corpus():
    """The small workload (K=20, V~3300, D=2000, ~200k tokens), regenerated
    from its seed; tests/test_golden.py checks it against the committed
    fixture's digests (tests/golden/small_chain.json)."""
    from gpupolyaurnlda_b200 import corpus
    return corpus.generate("small", seed=1)


@pytest.fixture(scope="session")
def gpu_lib():
    """Loads the in-tree CUDA library (fails loudly if it is missing)."""
    import torch
    assert torch.cuda.is_available(), "GPU test run without a CUDA device"
    import gpupolyaurnlda_b200 as g
    return g.lib()
