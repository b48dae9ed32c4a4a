"""gpupolyaurnlda_b200 -- Python binding of libGPUPolyaUrnLDA.so.

The library's C ABI (include/gpulda.h) is the reference's five-function FFI
(src/ffi.rs:15-31 <-> src/cu/train.cuh:41-45) plus gpulda_* additions.  This
module binds it with ctypes, with the same struct layouts as src/ffi.rs
(Args_FFI) and src/buffer.rs (Buffer), so tests and the benchmark call exactly
what the reference's Rust host calls.

There is no CPU fallback: importing `lib()` without the built library raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libGPUPolyaUrnLDA.so")

GPULDA_OK = 0
GPULDA_ERR_CUDA = 1
GPULDA_ERR_ARGS = 2
GPULDA_ERR_STATE = 3
GPULDA_ERR_BUFFER = 4
GPULDA_ERR_NOMEM = 5
GPULDA_ERR_DEVICE = 6
GPULDA_ERR_UNSUPPORTED = 7
GPULDA_FLAG_LOGLIK = 1
GPULDA_FLAG_HASHMAP = 2
GPULDA_MAX_K = 32768
GPULDA_MAX_DOC_LEN = 65535
POIS_TABLE_N, POIS_TABLE_W, LOGFAC_N = 64, 192, 256
KERNEL_TIME_NAMES = ("phi_draw", "prep", "alias_build", "doc_offsets", "z_sweep")
COUNTER_NAMES = ("tokens", "docs", "sparse_work", "sparse_draws", "launches")


class Args(C.Structure):
    """src/ffi.rs:4-13 Args_FFI / src/cu/train.cuh:13-21 Args."""

    _fields_ = [
        ("alpha", C.c_float),
        ("beta", C.c_float),
        ("K", C.c_uint32),
        ("V", C.c_uint32),
        ("C", C.POINTER(C.c_uint32)),
        ("buffer_size", C.c_uint32),
        ("max_D", C.c_uint32),
    ]


class Buffer(C.Structure):
    """src/buffer.rs:4-19 / src/cu/train.cuh:23-37."""

    _fields_ = [
        ("z", C.POINTER(C.c_uint32)),
        ("w", C.POINTER(C.c_uint32)),
        ("d", C.POINTER(C.c_uint32)),
        ("K_d", C.POINTER(C.c_uint32)),
        ("n_docs", C.c_uint32),
        ("n_tokens", C.c_uint32),
        ("gpu_z", C.c_void_p),
        ("gpu_w", C.c_void_p),
        ("gpu_d_len", C.c_void_p),
        ("gpu_d_idx", C.c_void_p),
        ("gpu_K_d", C.c_void_p),
        ("gpu_rng", C.c_void_p),
        ("stream", C.c_void_p),
    ]


class ExArgs(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("chain", C.c_uint32), ("flags", C.c_uint32)]


class Problem(C.Structure):
    """GpuldaProblem of include/gpulda_batch.h."""
    _fields_ = [
        ("alpha", C.c_float), ("beta", C.c_float), ("K", C.c_uint32), ("V", C.c_uint32),
        ("C", C.c_void_p), ("z", C.c_void_p), ("w", C.c_void_p), ("d_len", C.c_void_p),
        ("n_tokens", C.c_uint64), ("n_docs", C.c_uint32), ("flags", C.c_uint32),
        ("seed", C.c_uint64), ("chain", C.c_uint32), ("reserved", C.c_uint32),
    ]


class BatchShape(C.Structure):
    """GpuldaBatchShape of include/gpulda_batch.h."""
    _fields_ = [("z_warps_per_block", C.c_uint32), ("z_blocks_per_sm", C.c_uint32),
                ("phi_cells_per_block", C.c_uint32), ("reserved", C.c_uint32)]


class ServeArgs(C.Structure):
    """GpuldaServeArgs of include/gpulda_serve.h."""
    _fields_ = [("n_iter", C.c_uint32), ("mode", C.c_uint32), ("slots", C.c_uint32), ("max_batch", C.c_uint32),
                ("max_inflight", C.c_uint32), ("chain", C.c_uint32), ("seed", C.c_uint64),
                ("pool_bytes", C.c_uint64)]


SERVE_PERSISTENT = 0
SERVE_LAUNCH = 1


BATCH_BUCKETS = 4
BATCH_MAX_K = 2048

assert C.sizeof(Problem) == 80 and C.sizeof(BatchShape) == 16 and C.sizeof(ServeArgs) == 40
assert C.sizeof(Args) == 32 and Args.C.offset == 16
assert C.sizeof(Buffer) == 96 and Buffer.gpu_z.offset == 40

_U32P = C.POINTER(C.c_uint32)
_U64P = C.POINTER(C.c_uint64)
_F32P = C.POINTER(C.c_float)
_F64P = C.POINTER(C.c_double)

# name -> (restype, argtypes)
_SIGNATURES = {
    "initialize": (None, [C.POINTER(Args), C.POINTER(Buffer), C.c_uint32]),
    "sample_phi": (None, []),
    "sample_z_async": (None, [C.POINTER(Buffer)]),
    "sync_buffer": (None, [C.POINTER(Buffer)]),
    "cleanup": (None, [C.POINTER(Buffer), C.c_uint32]),
    "gpulda_last_error": (C.c_int, []),
    "gpulda_error_string": (C.c_char_p, [C.c_int]),
    "gpulda_set_fatal_errors": (None, [C.c_int]),
    "gpulda_initialize_ex": (C.c_int, [C.POINTER(Args), C.POINTER(Buffer), C.c_uint32, C.POINTER(ExArgs)]),
    "gpulda_set_stream": (C.c_int, [C.c_void_p]),
    "gpulda_pin_host": (C.c_int, [C.c_void_p, C.c_uint64, C.c_uint32]),
    "gpulda_set_token_offset": (C.c_int, [C.c_uint64]),
    "gpulda_count_table": (C.c_int, [C.POINTER(C.c_void_p), _U64P]),
    "gpulda_unpin_host": (C.c_int, [C.c_void_p]),
    "gpulda_loglik": (C.c_int, [_F64P, _U64P]),
    "gpulda_corpus_load": (C.c_int, [_U32P, _U32P, _U32P, C.c_uint32, C.c_uint64]),
    "gpulda_corpus_sweep": (C.c_int, [C.c_uint32]),
    "gpulda_corpus_read_z": (C.c_int, [_U32P]),
    "gpulda_corpus_count_rebuild": (C.c_int, [_F32P]),
    "gpulda_kernel_times": (C.c_int, [_F32P, C.c_int]),
    "gpulda_counters": (C.c_int, [_U64P, C.c_int]),
    "gpulda_debug_read": (C.c_int, [_U32P, _U32P, _U64P, _U64P, _U64P, _U32P]),
    "gpulda_debug_write_counts": (C.c_int, [_U32P]),
    "gpulda_debug_tables": (C.c_int, [_U32P, _F64P]),
    "gpulda_debug_philox": (C.c_int, [_U32P, C.c_uint32, C.c_uint32, C.c_uint32, _U32P]),
    "gpulda_debug_poisson": (C.c_int, [_U32P, _U64P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                       C.c_uint32, _U32P]),
    "gpulda_debug_alias": (C.c_int, [_U32P, C.c_uint32, _U64P]),
    "gpulda_sample_z_device_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64,
                                                 C.c_void_p]),
    # include/gpulda_batch.h
    "gpulda_batch_create": (C.c_int, [C.POINTER(Problem), C.c_uint32, C.POINTER(C.c_void_p)]),
    "gpulda_batch_destroy": (C.c_int, [C.c_void_p]),
    "gpulda_batch_sweep": (C.c_int, [C.c_void_p, C.c_uint32]),
    "gpulda_batch_sweep_async": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p]),
    "gpulda_batch_sync": (C.c_int, [C.c_void_p]),
    "gpulda_batch_read_z": (C.c_int, [C.c_void_p, C.c_uint32, _U32P]),
    "gpulda_batch_read_counts": (C.c_int, [C.c_void_p, C.c_uint32, _U32P]),
    "gpulda_batch_loglik": (C.c_int, [C.c_void_p, _F64P, _U64P]),
    "gpulda_batch_get_shapes": (C.c_int, [C.c_void_p, C.POINTER(BatchShape)]),
    "gpulda_batch_set_shapes": (C.c_int, [C.c_void_p, C.POINTER(BatchShape)]),
    "gpulda_batch_tune": (C.c_int, [C.c_void_p, C.c_char_p, _U32P]),
    "gpulda_batch_set_mode": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p]),
    "gpulda_batch_info": (C.c_int, [C.c_void_p, _U64P, C.c_int]),
    # include/gpulda_serve.h
    "gpulda_serve_create": (C.c_int, [C.POINTER(ServeArgs), C.POINTER(C.c_void_p)]),
    "gpulda_serve_create_from_phi": (C.c_int, [C.POINTER(ServeArgs), C.c_uint32, C.c_uint32, C.c_float, _U32P,
                                               C.POINTER(C.c_void_p)]),
    "gpulda_serve_destroy": (C.c_int, [C.c_void_p]),
    "gpulda_serve_submit": (C.c_int, [C.c_void_p, C.c_uint32, _U64P, _U32P, _U32P]),
    "gpulda_serve_progress": (C.c_int, [C.c_void_p]),
    "gpulda_serve_poll": (C.c_int, [C.c_void_p, C.c_uint32, _U64P, _F32P, _F64P, _U32P, _U64P, _U32P]),
    "gpulda_serve_drain": (C.c_int, [C.c_void_p]),
    "gpulda_serve_stats": (C.c_int, [C.c_void_p, _U64P, C.c_int]),
}

EXPORTED_SYMBOLS = tuple(_SIGNATURES)

_lib = None


def lib() -> C.CDLL:
    """Loads the in-tree library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run gpupolyaurnlda_b200/build.py (no CPU fallback exists)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class GpuldaError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        super().__init__(f"gpulda error {code} ({lib().gpulda_error_string(code).decode()}) {what}")
        self.code = code


def check(rc: int, what: str = "") -> None:
    if rc != GPULDA_OK:
        raise GpuldaError(rc, what)


def check_last(what: str = "") -> None:
    """For the void legacy entry points in non-fatal mode."""
    check(lib().gpulda_last_error(), what)


def ptr32(a: np.ndarray):
    assert a.dtype == np.uint32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_U32P)


def ptr64(a: np.ndarray):
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_U64P)


def make_args(alpha: float, beta: float, K: int, C_counts: np.ndarray, buffer_size: int, max_D: int) -> Args:
    return Args(alpha, beta, K, len(C_counts), ptr32(C_counts), buffer_size, max_D)


class Sampler:
    """A model held by the library (one per process, like the reference).

    Used by the tests and the benchmark; everything goes through the C ABI.
    """

    def __init__(self, alpha: float, beta: float, K: int, counts: np.ndarray, *, buffer_size: int = 1 << 25,
                 max_D: int = 16384, n_buffers: int = 1, seed: int = 0, chain: int = 0, flags: int = 0):
        self.L = lib()
        self.L.gpulda_set_fatal_errors(0)
        self.counts = np.ascontiguousarray(counts, dtype=np.uint32)
        self.K, self.V = int(K), int(len(self.counts))
        self.alpha, self.beta = float(alpha), float(beta)
        self.args = make_args(alpha, beta, K, self.counts, buffer_size, max_D)
        self.buffers = (Buffer * n_buffers)()
        self.n_buffers = n_buffers
        self.ex = ExArgs(seed, chain, flags)
        check(self.L.gpulda_initialize_ex(C.byref(self.args), self.buffers, n_buffers, C.byref(self.ex)), "initialize")
        self._live = True
        self._keep = []

    # --- reference protocol -------------------------------------------------
    def sample_phi(self) -> None:
        self.L.sample_phi()
        check_last("sample_phi")

    def sweep_buffer(self, i: int, z: np.ndarray, w: np.ndarray, d: np.ndarray, K_d: np.ndarray | None = None) -> None:
        b = self.buffers[i]
        b.z, b.w, b.d = ptr32(z), ptr32(w), ptr32(d)
        b.K_d = ptr32(K_d) if K_d is not None else C.cast(None, _U32P)
        b.n_docs, b.n_tokens = len(d), len(z)
        self._keep = [z, w, d, K_d]
        self.L.sample_z_async(C.byref(b))
        check_last("sample_z_async")
        self.L.sync_buffer(C.byref(b))
        check_last("sync_buffer")

    def close(self) -> None:
        if self._live:
            self.L.cleanup(self.buffers, self.n_buffers)
            self._live = False
            check_last("cleanup")

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # --- additions ------------------------------------------------------------
    def corpus_load(self, z: np.ndarray, w: np.ndarray, d_len: np.ndarray) -> None:
        self._corpus = (z, w, d_len)
        check(self.L.gpulda_corpus_load(ptr32(z), ptr32(w), ptr32(d_len), len(d_len), len(z)), "corpus_load")

    def corpus_sweep(self, n_iter: int = 1) -> None:
        check(self.L.gpulda_corpus_sweep(n_iter), "corpus_sweep")

    def corpus_count_rebuild(self) -> float:
        """Rebuilds the counts from the resident corpus's topics; returns the
        kernel's device time in ms."""
        ms = C.c_float()
        check(self.L.gpulda_corpus_count_rebuild(C.byref(ms)), "corpus_count_rebuild")
        return ms.value

    def corpus_z(self) -> np.ndarray:
        out = np.empty(len(self._corpus[0]), dtype=np.uint32)
        check(self.L.gpulda_corpus_read_z(ptr32(out)), "corpus_read_z")
        return out

    def set_stream(self, handle: int) -> None:
        check(self.L.gpulda_set_stream(C.c_void_p(handle)), "set_stream")

    def set_token_offset(self, first_token: int) -> None:
        """Global index of this process's first token (document sharding)."""
        check(self.L.gpulda_set_token_offset(first_token), "set_token_offset")

    def count_table(self):
        """The device count table n (K*V uint32, word-major) as a CUDA int32
        tensor sharing its memory (for an in-place all-reduce)."""
        import torch
        ptr = C.c_void_p()
        n = C.c_uint64()
        check(self.L.gpulda_count_table(C.byref(ptr), C.byref(n)), "count_table")

        class _Arr:
            __cuda_array_interface__ = {"shape": (n.value,), "typestr": "<i4", "data": (ptr.value, False),
                                        "version": 3, "strides": None}
        return torch.as_tensor(_Arr(), device="cuda")

    def loglik(self) -> tuple[float, int]:
        v = C.c_double()
        s = C.c_uint64()
        check(self.L.gpulda_loglik(C.byref(v), C.byref(s)), "loglik")
        return v.value, s.value

    def kernel_times(self) -> dict:
        a = (C.c_float * len(KERNEL_TIME_NAMES))()
        n = self.L.gpulda_kernel_times(a, len(a))
        return {KERNEL_TIME_NAMES[i]: float(a[i]) for i in range(n)}

    def counters(self) -> dict:
        a = np.zeros(len(COUNTER_NAMES), dtype=np.uint64)
        n = self.L.gpulda_counters(ptr64(a), len(a))
        return {COUNTER_NAMES[i]: int(a[i]) for i in range(n)}

    def read_state(self, n=True, q=True, alias=True, A=True, S=True, nnz=True) -> dict:
        K, V = self.K, self.V
        out = {}
        arrs = {
            "n": np.empty(K * V, np.uint32) if n else None,
            "q": np.empty(K * V, np.uint32) if q else None,
            "alias": np.empty(K * V, np.uint64) if alias else None,
            "A": np.empty(V, np.uint64) if A else None,
            "S": np.empty(K, np.uint64) if S else None,
            "nnz": np.empty(V, np.uint32) if nnz else None,
        }

        def p(a, f):
            return f(a) if a is not None else None

        check(self.L.gpulda_debug_read(p(arrs["n"], ptr32), p(arrs["q"], ptr32), p(arrs["alias"], ptr64),
                                       p(arrs["A"], ptr64), p(arrs["S"], ptr64), p(arrs["nnz"], ptr32)), "debug_read")
        for k, v in arrs.items():
            if v is not None:
                out[k] = v
        return out

    def write_counts(self, n: np.ndarray) -> None:
        n = np.ascontiguousarray(n, dtype=np.uint32)
        check(self.L.gpulda_debug_write_counts(ptr32(n)), "debug_write_counts")

    def tables(self) -> tuple[np.ndarray, np.ndarray]:
        cdf = np.empty(POIS_TABLE_N * POIS_TABLE_W, np.uint32)
        lfac = np.empty(LOGFAC_N, np.float64)
        check(self.L.gpulda_debug_tables(ptr32(cdf), lfac.ctypes.data_as(_F64P)), "debug_tables")
        return cdf, lfac

    def poisson(self, counts: np.ndarray, idx: np.ndarray, t: int, stream: int, key0: int = 0, key1: int = 0):
        counts = np.ascontiguousarray(counts, np.uint32)
        idx = np.ascontiguousarray(idx, np.uint64)
        out = np.empty(len(counts), np.uint32)
        check(self.L.gpulda_debug_poisson(ptr32(counts), ptr64(idx), len(counts), t, stream, key0, key1, ptr32(out)),
              "debug_poisson")
        return out


def device_philox(ctr: np.ndarray, key0: int, key1: int) -> np.ndarray:
    L = lib()
    ctr = np.ascontiguousarray(ctr, np.uint32).reshape(-1, 4)
    out = np.empty_like(ctr)
    check(L.gpulda_debug_philox(ptr32(ctr), len(ctr), key0, key1, ptr32(out)), "debug_philox")
    return out


def device_alias(q: np.ndarray) -> np.ndarray:
    L = lib()
    q = np.ascontiguousarray(q, np.uint32)
    out = np.empty(len(q), np.uint64)
    check(L.gpulda_debug_alias(ptr32(q), len(q), ptr64(out)), "debug_alias")
    return out
