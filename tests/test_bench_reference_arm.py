"""The CPU side of bench.py, with no GPU: the reference arm (`--impl
reference`) and the `cpu_baseline` sampler. The sampler times the
reference's own path (built from its sources into oracle/_ref) on the first
n_s points of the workload; n_s must stay a multiple of 8 (the reference's
self-term table is overrun otherwise, hilbertjoin/egojoin.h:178-195), and the
count it reports must be the FP64 oracle's count on that sample. The arm
prints exactly one JSON line, also when the reference fails."""
import argparse
import io
import json
import os
import sys
from contextlib import redirect_stdout

import numpy as np
import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402
from hilbertjoin_b200 import workloads as W  # noqa: E402

EPS = 2.279504  # the headline eps: one cell per dim, every pair evaluated
N_SMALL = 24_100  # not a multiple of 8: the sampler must cut it


def _have_ref():
    return oracle.pick_ref_binary(4, os.cpu_count() or 1) is not None


@pytest.fixture(scope="module")
def x_small():
    return W.uniform(N_SMALL, bench.DIM, bench.SEED, dtype=np.float32)


@pytest.mark.skipif(not _have_ref(), reason="reference build or AVX-512 host missing")
def test_sampler_times_reference_and_counts_match_oracle(x_small):
    s = bench.RefSampler(x_small, EPS, budget_s=0.05)
    assert s.kind == "reference" and s.kblock in (4, 16)
    assert s.n_s % 8 == 0 and s.n_s % bench.SAMPLE_ALIGN == 0 and bench.CAL_SAMPLE <= s.n_s <= N_SMALL
    r = s.run()
    assert r["count"] == oracle.self_count_brute(x_small[:s.n_s].astype(np.float64), EPS)
    assert set(bench.CPU_KEYS) <= set(r)
    assert r["kind"] == "reference" and r["avx512f"] is True and r["cores"] >= 1
    assert r["value"] == pytest.approx(s.n_s * (s.n_s - 1) / 2 / r["alg_s"])


def test_sampler_falls_back_to_port(x_small, monkeypatch):
    """Without a reference build the oracle's brute-force C port is timed,
    and the line says so."""
    monkeypatch.setattr(oracle, "pick_ref_binary", lambda *a, **k: None)
    s = bench.RefSampler(x_small, EPS, budget_s=0.05)
    assert s.kind == "port" and s.n_s % 8 == 0
    r = s.run()
    assert r["kind"] == "port" and "port" in r["sample"]
    assert r["count"] == oracle.self_count_brute(x_small[:s.n_s].astype(np.float64), EPS)


def _arm_line(monkeypatch, x):
    monkeypatch.setattr(bench, "workload", lambda n: (x, EPS))
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.run_reference(argparse.Namespace(steps=1, warmup=0, gpus=1))
    lines = [ln for ln in buf.getvalue().splitlines() if ln.strip()]
    assert len(lines) == 1, lines
    return json.loads(lines[0])


@pytest.mark.skipif(not _have_ref(), reason="reference build or AVX-512 host missing")
def test_reference_arm_line(x_small, monkeypatch):
    line = _arm_line(monkeypatch, x_small)
    assert line["impl"] == "reference" and line["metric"] == bench.METRIC and line["unit"] == bench.UNIT
    assert line["higher_is_better"] is True and line["steps"] == 1 and line["warmup"] == 0
    assert line["value"] > 0 and line["cpu_baseline"]["value"] == line["value"]
    assert line["cpu_baseline"]["kind"] == "reference"
    assert line["e2e"] == {"value": line["value"], "unit": bench.UNIT, "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["config"]["sample_points"] % 8 == 0


def test_reference_arm_reports_failure(x_small, monkeypatch):
    def boom(*a, **k):
        raise RuntimeError("planted failure")
    monkeypatch.setattr(bench, "RefSampler", boom)
    line = _arm_line(monkeypatch, x_small)
    assert line["impl"] == "reference" and "planted failure" in line["unavailable"]


def test_reference_arm_only_rank0(x_small, monkeypatch):
    """Under torchrun the ranks other than 0 exit without work or output."""
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setattr(bench, "workload", lambda n: pytest.fail("rank 1 built the workload"))
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.run_reference(argparse.Namespace(steps=1, warmup=0, gpus=2))
    assert buf.getvalue() == ""
