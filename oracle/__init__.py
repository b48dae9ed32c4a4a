"""CPU oracle of the Polya Urn LDA sweep -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs may
import this package, and only as the checker / the timed CPU reference; the
CUDA library never uses it.  The C++ restatement is oracle.cpp (each function
there cites the reference file:line it follows).

Parity is pinned by the reference's own unit-test vectors, restated for this
design in tests/test_oracle_kats.py (src/cu/test/test_topics.cu,
test_spalias.cu, test_polyaurn.cu, test_hashmap.cu), and by the published
Philox4x32-10 known-answer vectors.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .build import LIB, build_oracle, build_oracle_native

_U32P = C.POINTER(C.c_uint32)
_U64P = C.POINTER(C.c_uint64)
_F64P = C.POINTER(C.c_double)
_U8P = C.POINTER(C.c_uint8)

STREAM_INIT, STREAM_PHI, STREAM_Z = 1, 2, 3
POIS_N, POIS_W, LFAC_N = 64, 192, 256

_lib = None
_path = LIB


def use_native_build() -> str:
    """Switches this process to the -march=native build of the oracle (built
    here if needed; same results bit for bit).  For the timed CPU baseline;
    call before any other use of the oracle."""
    global _path
    assert _lib is None, "the oracle is already loaded"
    _path = build_oracle_native()
    return _path


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if _path == LIB and not os.path.exists(LIB):
            build_oracle()
        L = C.CDLL(_path)
        L.orc_philox.argtypes = [_U32P, C.c_uint32, C.c_uint32, C.c_uint32, _U32P]
        L.orc_tables.argtypes = [C.c_float, _U32P, _U8P, _F64P]
        L.orc_poisson.argtypes = [_U32P, _U64P, C.c_uint32, C.c_float, C.c_uint32, C.c_uint32, C.c_uint32,
                                  C.c_uint32, _U32P]
        L.orc_log.argtypes = [C.c_double]
        L.orc_log.restype = C.c_double
        L.orc_init_counts.argtypes = [C.c_uint32, C.c_uint32, C.c_float, _U32P, C.c_uint32, C.c_uint32, _U32P,
                                      C.c_int]
        L.orc_phi_step.argtypes = [C.c_uint32, C.c_uint32, C.c_float, _U32P, C.c_uint32, C.c_uint32, C.c_uint32,
                                   _U32P, _U64P, _U64P, _U64P, _U32P, C.c_int]
        L.orc_alias.argtypes = [_U32P, C.c_uint32, _U64P]
        L.orc_alias_items.argtypes = [_U32P, C.POINTER(C.c_uint16), C.c_uint32, _U64P]
        L.orc_doc_offsets.argtypes = [_U32P, C.c_uint32, _U64P]
        L.orc_z_sweep.argtypes = [C.c_uint32, C.c_uint32, C.c_float, _U32P, _U64P, _U64P, _U32P, _U32P, _U32P,
                                  _U32P, C.c_uint32, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, _U32P, _U64P,
                                  _F64P, _U32P, C.c_int]
        L.orc_alias_draw.argtypes = [_U64P, C.c_uint32, C.c_uint32, C.c_uint32]
        L.orc_alias_draw.restype = C.c_uint32
        L.orc_sparse_select.argtypes = [_U64P, C.c_uint32, C.c_uint32, _U64P]
        L.orc_sparse_select.restype = C.c_uint32
        L.orc_count_topics.argtypes = [_U32P, C.c_uint32, C.c_uint32, _U32P]
        L.orc_count_topics.restype = C.c_uint32
        L.orc_fold_in.argtypes = [C.c_uint32, C.c_uint32, C.c_float, _U32P, _U64P, _U64P, _U32P, _U32P, _U32P,
                                  _U64P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(C.c_float),
                                  _F64P, _U32P, _U32P, C.c_int]
        _lib = L
    return _lib


def _p32(a):
    assert a.dtype == np.uint32 and a.flags["C_CONTIGUOUS"], a.dtype
    return a.ctypes.data_as(_U32P)


def _p64(a):
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"], a.dtype
    return a.ctypes.data_as(_U64P)


def default_threads() -> int:
    return max(1, len(os.sched_getaffinity(0)))


def philox(ctr: np.ndarray, key0: int, key1: int) -> np.ndarray:
    ctr = np.ascontiguousarray(ctr, np.uint32).reshape(-1, 4)
    out = np.empty_like(ctr)
    lib().orc_philox(_p32(ctr), len(ctr), key0, key1, _p32(out))
    return out


def tables(beta: float):
    cdf = np.empty(POIS_N * POIS_W, np.uint32)
    guide = np.empty(POIS_N * 256, np.uint8)
    lfac = np.empty(LFAC_N, np.float64)
    lib().orc_tables(beta, _p32(cdf), guide.ctypes.data_as(_U8P), lfac.ctypes.data_as(_F64P))
    return cdf, guide, lfac


def poisson(counts, idx, beta: float, t: int, stream: int, key0: int = 0, key1: int = 0) -> np.ndarray:
    counts = np.ascontiguousarray(counts, np.uint32)
    idx = np.ascontiguousarray(idx, np.uint64)
    out = np.empty(len(counts), np.uint32)
    lib().orc_poisson(_p32(counts), _p64(idx), len(counts), beta, t, stream, key0, key1, _p32(out))
    return out


def det_log(x: float) -> float:
    return lib().orc_log(x)


def init_counts(K: int, counts: np.ndarray, beta: float, key0: int = 0, key1: int = 0, threads=None) -> np.ndarray:
    counts = np.ascontiguousarray(counts, np.uint32)
    V = len(counts)
    n = np.empty(K * V, np.uint32)
    lib().orc_init_counts(K, V, beta, _p32(counts), key0, key1, _p32(n), threads or default_threads())
    return n


def phi_step(K: int, V: int, beta: float, n: np.ndarray, t: int, key0: int = 0, key1: int = 0, threads=None) -> dict:
    n = np.ascontiguousarray(n, np.uint32)
    q = np.empty(K * V, np.uint32)
    al = np.empty(K * V, np.uint64)
    A = np.empty(V, np.uint64)
    S = np.empty(K, np.uint64)
    nnz = np.empty(V, np.uint32)
    lib().orc_phi_step(K, V, beta, _p32(n), t, key0, key1, _p32(q), _p64(al), _p64(A), _p64(S), _p32(nnz),
                       threads or default_threads())
    return {"q": q, "alias": al, "A": A, "S": S, "nnz": nnz}


def alias(q: np.ndarray) -> np.ndarray:
    q = np.ascontiguousarray(q, np.uint32)
    out = np.empty(len(q), np.uint64)
    lib().orc_alias(_p32(q), len(q), _p64(out))
    return out


def alias_items(q: np.ndarray, keys: np.ndarray) -> np.ndarray:
    """Alias table over len(q) items whose topics are `keys`."""
    q = np.ascontiguousarray(q, np.uint32)
    keys = np.ascontiguousarray(keys, np.uint16)
    out = np.empty(len(q), np.uint64)
    lib().orc_alias_items(_p32(q), keys.ctypes.data_as(C.POINTER(C.c_uint16)), len(q), _p64(out))
    return out


def live_alias_entries(alias: np.ndarray, nnz: np.ndarray, K: int) -> np.ndarray:
    """The entries a model uses: the first nnz[w] of each word's row."""
    V = len(nnz)
    mask = np.arange(K)[None, :] < nnz.astype(np.int64)[:, None]
    return alias.reshape(V, K)[mask]


def alias_draw(table: np.ndarray, r_slot: int, r_keep: int) -> int:
    table = np.ascontiguousarray(table, np.uint64)
    return int(lib().orc_alias_draw(_p64(table), len(table), r_slot, r_keep))


def sparse_select(mass: np.ndarray, r: int) -> tuple[int, np.ndarray]:
    mass = np.ascontiguousarray(mass, np.uint64)
    prefix = np.empty(len(mass), np.uint64)
    i = lib().orc_sparse_select(_p64(mass), len(mass), r, _p64(prefix))
    return int(i), prefix


def count_topics(z: np.ndarray, K: int) -> tuple[int, np.ndarray]:
    z = np.ascontiguousarray(z, np.uint32)
    counts = np.empty(K, np.uint32)
    d = lib().orc_count_topics(_p32(z), len(z), K, _p32(counts))
    return int(d), counts


def doc_offsets(d_len: np.ndarray) -> np.ndarray:
    d_len = np.ascontiguousarray(d_len, np.uint32)
    out = np.empty(len(d_len), np.uint64)
    lib().orc_doc_offsets(_p32(d_len), len(d_len), _p64(out))
    return out


def z_sweep(K: int, V: int, alpha: float, phi: dict, w: np.ndarray, z: np.ndarray, d_len: np.ndarray, t: int,
            tok_base: int = 0, key0: int = 0, key1: int = 0, n_out: np.ndarray | None = None, want_ll=False,
            threads=None) -> dict:
    """Sweeps z in place; returns counts n (word-major), stats, loglik, K_d."""
    w = np.ascontiguousarray(w, np.uint32)
    d_len = np.ascontiguousarray(d_len, np.uint32)
    assert z.dtype == np.uint32 and z.flags["C_CONTIGUOUS"]
    if n_out is None:
        n_out = np.zeros(K * V, np.uint32)
    stats = np.zeros(4, np.uint64)
    ll = np.zeros(2, np.float64)
    K_d = np.empty(len(d_len), np.uint32)
    lib().orc_z_sweep(K, V, alpha, _p32(phi["q"]), _p64(phi["alias"]), _p64(phi["A"]), _p32(phi["nnz"]), _p32(w),
                      _p32(z), _p32(d_len), len(d_len), tok_base, t, key0, key1, _p32(n_out), _p64(stats),
                      ll.ctypes.data_as(_F64P) if want_ll else None, _p32(K_d), threads or default_threads())
    return {"n": n_out, "stats": stats, "ll": float(ll[0]), "ll_skipped": int(ll[1]), "K_d": K_d}


def fold_in(K: int, V: int, alpha: float, phi: dict, w: np.ndarray, lengths: np.ndarray, ids: np.ndarray,
            n_iter: int, seed: int = 0, chain: int = 0, threads=None) -> dict:
    """Fold-in of new documents against a fixed model (phi: q, alias, A, nnz
    of a Phi step): theta (float32, n x K), loglik, skipped, final topics."""
    w = np.ascontiguousarray(w, np.uint32)
    lengths = np.ascontiguousarray(lengths, np.uint32)
    ids = np.ascontiguousarray(ids, np.uint64)
    n = len(lengths)
    theta = np.empty(n * K, np.float32)
    ll = np.empty(n, np.float64)
    skipped = np.empty(n, np.uint32)
    z = np.empty(max(1, len(w)), np.uint32)
    lib().orc_fold_in(K, V, alpha, _p32(phi["q"]), _p64(phi["alias"]), _p64(phi["A"]), _p32(phi["nnz"]), _p32(w),
                      _p32(lengths), _p64(ids), n, seed & 0xffffffff, chain, n_iter,
                      theta.ctypes.data_as(C.POINTER(C.c_float)), ll.ctypes.data_as(_F64P), _p32(skipped), _p32(z),
                      threads or default_threads())
    return {"theta": theta.reshape(n, K), "ll": ll, "skipped": skipped, "z": z[:len(w)]}


class Chain:
    """Whole iterations on the CPU: the reference's stage order
    (src/cu/train.cu:137-172) -- Phi step from the previous counts, then one
    z sweep that rebuilds the counts."""

    def __init__(self, K, alpha, beta, counts, seed=0, chain=0, threads=None):
        self.K, self.alpha, self.beta = K, alpha, beta
        self.counts = np.ascontiguousarray(counts, np.uint32)
        self.V = len(self.counts)
        self.key0, self.key1 = seed, chain
        self.threads = threads
        self.n = init_counts(K, self.counts, beta, seed, chain, threads)
        self.t = -1
        self.phi = None

    def sample_phi(self):
        self.t += 1
        self.phi = phi_step(self.K, self.V, self.beta, self.n, self.t, self.key0, self.key1, self.threads)
        self.n = np.zeros(self.K * self.V, np.uint32)
        self.tok_base = 0

    def sweep(self, w, z, d_len, want_ll=False):
        r = z_sweep(self.K, self.V, self.alpha, self.phi, w, z, d_len, self.t, self.tok_base, self.key0, self.key1,
                    self.n, want_ll, self.threads)
        self.tok_base += int(np.asarray(d_len, np.uint64).sum())
        return r
