"""CPU-only checks of the drop-in boundary and the host logic (no GPU calls).

* libGPUPolyaUrnLDA.so loads and exports every entry point include/*.h
  declares, with the reference's unmangled names (src/cu/train.cuh:41-45).
* Args / Buffer layouts equal the reference's repr(C) structs
  (src/ffi.rs:4-13, src/buffer.rs:4-19).
* The host-built Poisson tables of the library equal the oracle's.
* The buffer-filling rules of the train loop twin (src/train.rs:20-58).
* The reference's file formats (src/preprocess.rs:42-72, src/output.rs:27-62).
"""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import gpupolyaurnlda_b200 as g
from gpupolyaurnlda_b200 import corpus
from gpupolyaurnlda_b200.train import GpuldaError, fill_sizes, iterate_buffers

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_functions():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:void|int|const char\*)\s+\*?(\w+)\s*\(", text, flags=re.M)
    return names


@pytest.fixture(scope="module")
def built():
    from gpupolyaurnlda_b200.build import build_library
    build_library()
    return C.CDLL(g.LIB_PATH)


def test_library_exports_every_declared_symbol(built):
    names = _header_functions()
    assert {"initialize", "sample_phi", "sample_z_async", "sync_buffer", "cleanup"} <= set(names)
    for n in names:
        assert hasattr(built, n), f"{n} declared in include/ but not exported"
    assert set(names) == set(g.EXPORTED_SYMBOLS)


def test_reference_symbols_are_unmangled():
    out = subprocess.run(["nm", "-D", "--defined-only", g.LIB_PATH], capture_output=True, text=True).stdout
    syms = {line.split()[-1] for line in out.splitlines() if line.strip()}
    for n in ("initialize", "sample_phi", "sample_z_async", "sync_buffer", "cleanup"):
        assert n in syms


def test_struct_layouts_match_reference():
    # Args_FFI: f32 alpha, f32 beta, u32 K, u32 V, *const c_void C, u32 buffer_size, u32 max_D
    assert C.sizeof(g.Args) == 32
    assert [g.Args.alpha.offset, g.Args.beta.offset, g.Args.K.offset, g.Args.V.offset, g.Args.C.offset,
            g.Args.buffer_size.offset, g.Args.max_D.offset] == [0, 4, 8, 12, 16, 24, 28]
    # Buffer: 4 host pointers, n_docs, n_tokens, 7 library-owned slots
    assert C.sizeof(g.Buffer) == 96
    assert [g.Buffer.z.offset, g.Buffer.K_d.offset, g.Buffer.n_docs.offset, g.Buffer.n_tokens.offset,
            g.Buffer.gpu_z.offset, g.Buffer.stream.offset] == [0, 24, 32, 36, 40, 88]


def test_host_tables_equal_oracle_tables(tmp_path, oracle_lib):
    src = tmp_path / "dump.cpp"
    src.write_text(r'''
#include <cstdio>
#include <vector>
#include "tables.h"
int main(int argc, char** argv) {
  float beta = (float)atof(argv[1]);
  std::vector<uint32_t> cdf(64 * 192); std::vector<uint8_t> guide(64 * 256); std::vector<double> lf(256);
  gpulda::build_poisson_tables(beta, 64, 192, cdf.data(), guide.data());
  gpulda::build_log_factorials(256, lf.data());
  fwrite(cdf.data(), 4, cdf.size(), stdout); fwrite(guide.data(), 1, guide.size(), stdout);
  fwrite(lf.data(), 8, lf.size(), stdout); return 0;
}
''')
    exe = tmp_path / "dump"
    subprocess.run(["g++", "-O2", "-ffp-contract=off", "-include", "cstdlib", "-I",
                    os.path.join(ROOT, "gpupolyaurnlda_b200", "csrc"), str(src), "-o", str(exe)], check=True)
    for beta in (0.01, 0.1, 0.0, 0.5):
        raw = subprocess.run([str(exe), repr(beta)], capture_output=True, check=True).stdout
        cdf = np.frombuffer(raw[:64 * 192 * 4], np.uint32)
        guide = np.frombuffer(raw[64 * 192 * 4:64 * 192 * 4 + 64 * 256], np.uint8)
        lf = np.frombuffer(raw[64 * 192 * 4 + 64 * 256:], np.float64)
        ocdf, oguide, olf = oracle_lib.tables(beta)
        assert (cdf == ocdf).all() and (guide == oguide).all() and (lf == olf).all()


def test_fill_buffer_rules():
    d = np.array([5, 3, 7, 2, 0, 4], np.uint32)
    # a zero-length document ends the corpus, as in src/train.rs:31
    assert fill_sizes(d, 0, 100, 100) == (4, 17)
    assert fill_sizes(d, 0, 100, 2) == (2, 8)      # max_D
    assert fill_sizes(d, 0, 10, 100) == (2, 8)     # buffer_size
    assert fill_sizes(d, 4, 100, 100) == (0, 0)
    with pytest.raises(GpuldaError):
        fill_sizes(np.array([11], np.uint32), 0, 10, 100)
    z = np.arange(17, dtype=np.uint32)
    bufs = list(iterate_buffers(z, z, d, d, 9, 100))
    assert [len(b[2]) for b in bufs] == [2, 2] and [len(b[0]) for b in bufs] == [8, 9]


def test_reference_file_formats(tmp_path):
    c = corpus.generate("small", seed=3, D=50)
    paths = corpus.write_files(c, str(tmp_path))
    assert (np.fromfile(paths["z"], "<u4") == c.z).all()
    assert (np.fromfile(paths["w"], "<u4") == c.w).all()
    assert (np.fromfile(paths["d"], "<u4") == c.d_len).all()
    assert (np.fromfile(paths["k_d"], "<u4") == c.k_d()).all()
    counts = corpus.read_counts(paths["c"])
    assert (counts == c.counts).all()
    assert (np.diff(counts.astype(np.int64)) <= 0).all(), "ids ranked by descending count"
    assert (np.bincount(c.w, minlength=c.V) == counts).all()
    out = tmp_path / "out.txt"
    corpus.write_output(paths["z"], paths["w"], paths["d"], paths["c"], str(out))
    lines = out.read_text().split("\n")[:-1]
    assert len(lines) == c.n_docs
    first = lines[0].rstrip("\t").split("\t")
    assert len(first) == c.d_len[0]
    tok, topic = first[0].rsplit(":", 1)
    assert tok == f"w{c.w[0]}" and int(topic) == c.z[0]


def test_gpulda_train_binary_parses_reference_flags(built):
    exe = os.path.join(ROOT, "gpupolyaurnlda_b200", "gpulda_train")
    assert os.path.exists(exe)
    r = subprocess.run([exe, "--no_such_flag"], capture_output=True, text=True)
    assert r.returncode == 2 and "unknown flag" in r.stderr
    # --help lists every flag of src/args.rs:16-61 with the reference's defaults
    r = subprocess.run([exe, "--help"], capture_output=True, text=True)
    assert r.returncode == 0
    for flag, default in [("--alpha", "0.1"), ("--beta", "0.1"), ("--K", "100"), ("--buffer_size", "33554432"),
                          ("--max_D", "16384"), ("--n_mc", "1"), ("--seed", "0"), ("--input", "data/small.txt"),
                          ("--output", "output/small.txt"), ("--z_temp_file", "temp/z.bin"),
                          ("--w_temp_file", "temp/w.bin"), ("--d_temp_file", "temp/d.bin"),
                          ("--K_d_temp_file", "temp/k_d.bin"), ("--c_temp_file", "temp/c.txt")]:
        assert flag in r.stdout and default in r.stdout, flag


def test_batch_problem_layout():
    # GpuldaProblem of include/gpulda_batch.h
    P = g.Problem
    assert C.sizeof(P) == 80
    assert [P.alpha.offset, P.beta.offset, P.K.offset, P.V.offset, P.C.offset, P.z.offset, P.w.offset,
            P.d_len.offset, P.n_tokens.offset, P.n_docs.offset, P.flags.offset, P.seed.offset,
            P.chain.offset] == [0, 4, 8, 12, 16, 24, 32, 40, 48, 56, 60, 64, 72]


def test_batch_create_rejects_bad_problems_before_any_device_call(built):
    """Validation runs on the host before anything touches a device, so the
    rejected cases need no GPU."""
    from gpupolyaurnlda_b200.batch import BatchChains, ProblemSpec
    counts = np.array([3, 2, 1], np.uint32)
    ok = dict(alpha=0.1, beta=0.01, K=4, counts=counts, z=np.array([0, 1, 2], np.uint32),
              w=np.array([0, 1, 2], np.uint32), d_len=np.array([2, 1], np.uint32))
    cases = [
        (dict(K=4096), 7),                                        # above GPULDA_BATCH_MAX_K
        (dict(K=0), 2),
        (dict(alpha=0.0), 2),
        (dict(w=np.array([0, 1, 3], np.uint32)), 2),              # word id >= V
        (dict(z=np.array([0, 1, 4], np.uint32)), 2),              # topic >= K
        (dict(d_len=np.array([2, 2], np.uint32)), 2),             # lengths do not sum to n_tokens
        (dict(d_len=np.array([70000], np.uint32), z=np.zeros(70000, np.uint32),
              w=np.zeros(70000, np.uint32)), 7),                  # document above GPULDA_MAX_DOC_LEN
    ]
    for change, code in cases:
        spec = ProblemSpec(**{**ok, **change})
        with pytest.raises(GpuldaError) as e:
            BatchChains([ProblemSpec(**ok), spec])
        assert e.value.code == code, change
    with pytest.raises(GpuldaError) as e:
        BatchChains([])
    assert e.value.code == 2
