"""The allocation-free sweep, gpulda_sample_z_device_noalloc.

That entry point serves callers that may not allocate device memory when they
call: an application that owns every device byte through its own pool, a
service that allocates nothing once it is serving, or work issued where
cudaMalloc is not permitted.  It keeps its scratch in a fixed device array of
the library instead of allocating.  Here it must give exactly what the
existing buffer entry point (sample_z_async / sync_buffer) gives on the same
model state -- topics and counts bit for bit, log-likelihood within 1e-4
relative, the tolerances of the other parity tests -- on two calls in a row,
and it must refuse more documents than its scratch holds.

This file is collected last so that a run stopping at the first failure has
run every other test before it.
"""
import numpy as np
import pytest
import torch

import gpupolyaurnlda_b200 as g
from gpupolyaurnlda_b200 import corpus

pytestmark = pytest.mark.gpu

SEED = 21


def _device_u32(a: np.ndarray) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a, np.uint32).view(np.int32)).cuda()


def test_noalloc_sweep_matches_buffer_entry_point(gpu_lib):
    c = corpus.generate("small", seed=2, D=300)
    # existing entry point: host buffers through sample_z_async / sync_buffer
    z = c.z.copy()
    expected = []
    with g.Sampler(c.alpha, c.beta, c.K, c.counts, buffer_size=c.n_tokens, max_D=c.n_docs, seed=SEED,
                   flags=g.GPULDA_FLAG_LOGLIK) as s:
        for _ in range(2):
            s.sample_phi()
            s.sweep_buffer(0, z, c.w, c.d_len, c.k_d())
            n = s.read_state(q=False, alias=False, A=False, S=False, nnz=False)["n"]
            expected.append((z.copy(), n, s.loglik()[0]))
    # allocation-free entry point: the same documents already in device memory
    dz, dw, dd = _device_u32(c.z), _device_u32(c.w), _device_u32(c.d_len)
    torch.cuda.synchronize()
    L = g.lib()
    with g.Sampler(c.alpha, c.beta, c.K, c.counts, buffer_size=c.n_tokens, max_D=c.n_docs, seed=SEED,
                   flags=g.GPULDA_FLAG_LOGLIK) as s:
        for i in range(2):
            s.sample_phi()
            rc = L.gpulda_sample_z_device_noalloc(dz.data_ptr(), dw.data_ptr(), dd.data_ptr(), c.n_docs,
                                                  c.n_tokens, None)
            assert rc == g.GPULDA_OK
            torch.cuda.synchronize()
            z_now = dz.cpu().numpy().view(np.uint32)
            assert (z_now == expected[i][0]).all(), f"call {i}: topics differ"
            n = s.read_state(q=False, alias=False, A=False, S=False, nnz=False)["n"]
            assert (n == expected[i][1]).all(), f"call {i}: counts differ"
            ll = s.loglik()[0]
            assert abs(ll - expected[i][2]) <= 1e-4 * abs(expected[i][2])
        # more documents than the fixed scratch holds: refused, nothing launched
        rc = L.gpulda_sample_z_device_noalloc(dz.data_ptr(), dw.data_ptr(), dd.data_ptr(), 1048576 + 1,
                                              c.n_tokens, None)
        assert rc == g.GPULDA_ERR_UNSUPPORTED
        assert L.gpulda_last_error() == g.GPULDA_ERR_UNSUPPORTED


def _large_k_corpus():
    import dataclasses
    wl = dataclasses.replace(corpus.WORKLOADS["large_k10000"], K=4096, V=3000, D=400)
    return corpus.generate(wl, seed=6)


@pytest.mark.parametrize("K", [20, 4096])
def test_noalloc_on_caller_stream_without_host_sync(gpu_lib, K):
    """Three iterations whose sweeps run on a stream of the caller's (a torch
    stream, not the library's), with no host synchronization between a sweep
    and the next sample_phi: the Phi step must wait for the sweep on the GPU.
    At K=4096 the large-K store is used.  The chain must equal the buffer
    entry point's, topics and counts bit for bit, log-likelihood within 1e-4
    relative."""
    c = corpus.generate("small", seed=3, D=300) if K == 20 else _large_k_corpus()
    assert c.K == K
    n_iter = 3
    z = c.z.copy()
    with g.Sampler(c.alpha, c.beta, c.K, c.counts, buffer_size=c.n_tokens, max_D=c.n_docs, seed=SEED,
                   flags=g.GPULDA_FLAG_LOGLIK) as s:
        for _ in range(n_iter):
            s.sample_phi()
            s.sweep_buffer(0, z, c.w, c.d_len, c.k_d())
        n_want = s.read_state(q=False, alias=False, A=False, S=False, nnz=False)["n"]
        ll_want = s.loglik()[0]
    dz, dw, dd = _device_u32(c.z), _device_u32(c.w), _device_u32(c.d_len)
    torch.cuda.synchronize()
    st = torch.cuda.Stream()
    L = g.lib()
    with g.Sampler(c.alpha, c.beta, c.K, c.counts, buffer_size=c.n_tokens, max_D=c.n_docs, seed=SEED,
                   flags=g.GPULDA_FLAG_LOGLIK) as s:
        for _ in range(n_iter):
            s.sample_phi()
            rc = L.gpulda_sample_z_device_noalloc(dz.data_ptr(), dw.data_ptr(), dd.data_ptr(), c.n_docs,
                                                  c.n_tokens, st.cuda_stream)
            assert rc == g.GPULDA_OK
        st.synchronize()
        assert (dz.cpu().numpy().view(np.uint32) == z).all(), "topics differ from the buffer entry point"
        n = s.read_state(q=False, alias=False, A=False, S=False, nnz=False)["n"]
        assert (n == n_want).all(), "counts differ from the buffer entry point"
        ll = s.loglik()[0]
        assert abs(ll - ll_want) <= 1e-4 * abs(ll_want)
