"""The two executables: the reference's flags and one-line output format
(main.cpp:122, mainJoin.cpp:139), inputs from CSV, FP64 .bin and FP32 .f32."""
import os
import subprocess

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "hilbertjoin_b200", "bin")


@pytest.fixture(scope="module")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def run(args):
    r = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return r.stdout.strip().splitlines()[-1].split(";")


@pytest.mark.parametrize("fmt", ["csv", "bin", "f32"])
@pytest.mark.parametrize("form", ["plain", "tf32", "fp16"])
def test_self_cli(gpu, tmp_path, fmt, form):
    x = np.random.default_rng(4).random((3000, 16))
    if fmt == "f32":
        x = x.astype(np.float32).astype(np.float64)
    p = tmp_path / f"x.{fmt}"
    if fmt == "csv":
        with open(p, "w") as f:
            f.write("% a comment line\n")
            for row in x:
                f.write(",".join(repr(float(v)) for v in row) + "\n")
    elif fmt == "bin":
        x.tofile(p)
    else:
        x.astype(np.float32).tofile(p)
    eps = 0.55
    out = run([os.path.join(BIN, "hilbertSelfJoinCardinality"), "-n", "3000", "-e", str(eps), "-d", "16", "-f",
               str(p), "-t", "64", "-F", form])
    assert len(out) == 15  # N;D;JPPP;THREADS;EPSILON;STRIPES;KBLOCK;TIME;ALGTIME;SORTTIME;INDEXTIME;REORDERTIME;COUNTS;LOADPERCENT;WH
    assert out[0] == "3000" and out[1] == "16" and out[5] == "14"
    want = oracle.self_count_brute(x, eps)
    assert int(out[12]) == want
    assert abs(float(out[2]) - want / 3000) < 1e-5


def test_join_cli_reads_g(gpu, tmp_path):
    a = np.random.default_rng(5).random((2000, 8))
    b = np.random.default_rng(6).random((2500, 8))
    a.tofile(tmp_path / "a.bin")
    b.tofile(tmp_path / "b.bin")
    eps = 0.3
    out = run([os.path.join(BIN, "hilbertJoinCardinality"), "-n", "2000", "-m", "2500", "-e", str(eps), "-d", "8",
               "-f", str(tmp_path / "a.bin"), "-g", str(tmp_path / "b.bin")])
    assert len(out) == 16
    assert int(out[13]) == oracle.join_count_brute(a, b, eps)


def test_cli_generated_data_and_errors(gpu, tmp_path):
    out = run([os.path.join(BIN, "hilbertSelfJoinCardinality"), "-n", "20000", "-e", "0.2", "-d", "64"])
    assert out[12] == "0"  # the README example shape: no pairs at eps 0.2 in 64-d
    r = subprocess.run([os.path.join(BIN, "hilbertSelfJoinCardinality"), "-n", "10", "-e", "0.2", "-d", "4", "-f",
                        str(tmp_path / "missing.bin")], capture_output=True, text=True)
    assert r.returncode != 0 and "does not exist" in r.stderr
    (tmp_path / "short.bin").write_bytes(b"\0" * 64)
    r = subprocess.run([os.path.join(BIN, "hilbertSelfJoinCardinality"), "-n", "10", "-e", "0.2", "-d", "4", "-f",
                        str(tmp_path / "short.bin")], capture_output=True, text=True)
    assert r.returncode != 0
