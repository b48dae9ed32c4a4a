"""The C++ twin of the reference's command line (src/main.rs): preprocess
(src/preprocess.rs:16-72) and output (src/output.rs:27-62) on the CPU, and the
whole text -> topics pipeline on the GPU, where the double-buffered, pinned
streaming loop must give the topics of the reference's serial loop bit for
bit."""
import os
import subprocess

import numpy as np
import pytest

from gpupolyaurnlda_b200 import corpus

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "gpupolyaurnlda_b200", "gpulda_train")


@pytest.fixture(scope="module")
def exe():
    from gpupolyaurnlda_b200.build import build_library
    build_library()
    return EXE


def _text_corpus(path, n_docs=60, seed=3):
    """Lines "docno:i<TAB>X<TAB>tokens" as the reference's input
    (src/preprocess.rs:12-14), Zipf-ish words, some repeated."""
    rng = np.random.default_rng(seed)
    vocab = [f"tok{i}" for i in range(40)] + ["alpha", "beta", "gamma"]
    p = 1.0 / np.arange(1, len(vocab) + 1)
    p /= p.sum()
    docs = []
    with open(path, "w") as f:
        for i in range(n_docs):
            L = int(rng.integers(1, 30))
            toks = [vocab[j] for j in rng.choice(len(vocab), L, p=p)]
            docs.append(toks)
            f.write(f"docno:{i}\tX\t{' '.join(toks)}\n")
    return docs


def _paths(tmp, tag=""):
    return {k: str(tmp / f"{k}{tag}") for k in ("z.bin", "w.bin", "d.bin", "k_d.bin", "c.txt", "out.txt")}


def _flags(p, extra=()):
    return ["--z_temp_file", p["z.bin"], "--w_temp_file", p["w.bin"], "--d_temp_file", p["d.bin"],
            "--K_d_temp_file", p["k_d.bin"], "--c_temp_file", p["c.txt"], "--output", p["out.txt"], *extra]


def test_preprocess_writes_reference_files(exe, tmp_path):
    docs = _text_corpus(tmp_path / "in.txt")
    p = _paths(tmp_path)
    r = subprocess.run([exe, "--phases", "preprocess", "--input", str(tmp_path / "in.txt"), "--K", "7",
                        "--seed", "5", *_flags(p)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    names = corpus.read_names(p["c.txt"])
    counts = corpus.read_counts(p["c.txt"])
    assert (np.diff(counts.astype(np.int64)) <= 0).all()  # ids by descending count
    z = np.fromfile(p["z.bin"], "<u4")
    w = np.fromfile(p["w.bin"], "<u4")
    d = np.fromfile(p["d.bin"], "<u4")
    kd = np.fromfile(p["k_d.bin"], "<u4")
    assert list(d) == [len(t) for t in docs]
    assert [names[int(i)] for i in w] == [t for doc in docs for t in doc]
    assert (np.bincount(w, minlength=len(counts)) == counts).all()
    assert z.max() < 7
    offs = np.concatenate([[0], np.cumsum(d.astype(np.int64))]).astype(np.int64)
    assert list(kd) == [len(set(z[offs[i]:offs[i + 1]])) for i in range(len(d))]
    # seeded: the same seed gives the same initial topics
    p2 = _paths(tmp_path, ".2")
    subprocess.run([exe, "--phases", "preprocess", "--input", str(tmp_path / "in.txt"), "--K", "7", "--seed", "5",
                    *_flags(p2)], check=True, capture_output=True)
    assert (np.fromfile(p2["z.bin"], "<u4") == z).all()


def test_output_matches_python_twin(exe, tmp_path):
    _text_corpus(tmp_path / "in.txt")
    p = _paths(tmp_path)
    subprocess.run([exe, "--phases", "preprocess,output", "--input", str(tmp_path / "in.txt"), "--K", "9",
                    *_flags(p)], check=True, capture_output=True)
    ref = tmp_path / "py_out.txt"
    corpus.write_output(p["z.bin"], p["w.bin"], p["d.bin"], p["c.txt"], str(ref))
    assert open(p["out.txt"]).read() == ref.read_text()


def test_rejects_line_without_token_field(exe, tmp_path):
    (tmp_path / "bad.txt").write_text("docno:1\tX\tok tokens\nonly_one_field\n")
    r = subprocess.run([exe, "--phases", "preprocess", "--input", str(tmp_path / "bad.txt"), *_flags(_paths(tmp_path))],
                       capture_output=True, text=True)
    assert r.returncode != 0 and "line 2" in r.stderr


@pytest.mark.gpu
def test_pipeline_double_buffered_pinned_equals_serial(exe, tmp_path, gpu_lib):
    _text_corpus(tmp_path / "in.txt", n_docs=400, seed=8)
    outs = []
    for tag, extra in (("s", []), ("db", ["--double_buffer", "1", "--pin", "1"])):
        p = _paths(tmp_path, tag)
        r = subprocess.run([exe, "--input", str(tmp_path / "in.txt"), "--K", "12", "--n_mc", "4", "--seed", "2",
                            "--buffer_size", "500", "--max_D", "37", *_flags(p, extra)], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        outs.append((np.fromfile(p["z.bin"], "<u4"), open(p["out.txt"]).read()))
    assert (outs[0][0] == outs[1][0]).all()
    assert outs[0][1] == outs[1][1]
    assert outs[0][0].max() < 12
