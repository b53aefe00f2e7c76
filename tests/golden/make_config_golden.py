"""Generates tests/golden/config_counts.json: the pair counts of the benchmark
configurations at their stated sizes.

The configurations (``hilbertjoin_b200.workloads.CONFIGS``) are regenerated
from their seeds at test time; only counts and timings are stored. For every
configuration this script records

* ``oracle_count``: the FP64 count of ``oracle/hj_oracle.c`` -- the brute-force
  count over all pairs where that finishes in about an hour on 8 cores
  (``oracle_method: "brute"``), else the oracle's EGO + stripe count, whose
  candidate ranges provably hold every pair the FP64 test accepts
  (``oracle_method: "ego"``);
* ``ref_count``: the count of the hilbertJoin reference built from its own
  sources (``oracle/build_ref.sh``) through ``test_ego_loop3_macro`` /
  ``test_ego_loop3_noself`` (hilbertjoin/egojoin.cpp:777, :840). The
  reference needs d % 8 == 0 for its vector loads, so d = 20 and d = 28 run
  zero-padded to 24 and 32 (``ref_pad_to``); zero columns change no cell and
  no distance. All configured n are multiples of 8, the reference's valid
  domain (its self-term table overruns for other n, egojoin.h:178-195);
* the wall times of both, so that the cost of re-running is known.

Run from the repository root (needs the reference sources for oracle/_ref):

    python tests/golden/make_config_golden.py [--only NAME ...] [--threads T]

The FP32 configurations are widened exactly to FP64 before counting, so both
counters see the values the engine sees.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from hilbertjoin_b200 import workloads as W  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "config_counts.json")

# oracle method per configuration: brute force where it is affordable
METHOD = {
    "cfg1_self_200k_d64": "brute",
    "cfg2_join_200k_d20": "brute",
    "cfg2_join_200k_d20_nbrs20": "brute",
    "cfg3_self_1M_d64_nbrs32": "brute",
    "cfg4_self_4M_d28_gmm64_nbrs100": "ego",
}


def pad(x: np.ndarray, to: int) -> np.ndarray:
    if x.shape[1] >= to:
        return x
    return np.concatenate([x, np.zeros((x.shape[0], to - x.shape[1]))], axis=1)


def run(name: str, threads: int) -> dict:
    c = W.CONFIGS[name]
    a, b, eps = W.config_sets(name)
    a = a.astype(np.float64)
    b = None if b is None else b.astype(np.float64)
    rec = {"eps": eps, "n": c["n"], "d": c["d"], "kind": c["kind"]}
    if b is not None:
        rec["m"] = c["m"]
    meth = METHOD[name]
    t = time.time()
    if c["kind"] == "self":
        if meth == "brute":
            oc = oracle.self_count_brute(a, eps, threads=threads)
        else:
            oc, cand = oracle.self_count_ego(a, eps, active_dims=3, threads=threads)
            rec["oracle_candidates"] = cand
    else:
        if meth == "brute":
            oc = oracle.join_count_brute(a, b, eps, threads=threads)
        else:
            oc, cand = oracle.join_count_ego(a, b, eps, active_dims=2, threads=threads)
            rec["oracle_candidates"] = cand
    rec.update(oracle_count=int(oc), oracle_method=meth, oracle_s=round(time.time() - t, 1))
    print(f"{name}: oracle {oc} ({meth}, {rec['oracle_s']} s)", flush=True)

    ref_pad = (c["d"] + 7) // 8 * 8
    if oracle.pick_ref_binary(4, threads) is not None:
        t = time.time()
        if c["kind"] == "self":
            r = oracle.ref_self_count(pad(a, ref_pad), eps, stripes=14, kblock=4, threads=threads)
        else:
            r = oracle.ref_join_count(pad(a, ref_pad), pad(b, ref_pad), eps, kblock=4, threads=threads)
        rec.update(ref_count=int(r["count"]), ref_pad_to=ref_pad, ref_s=round(time.time() - t, 1),
                   ref_loadpercent=r["loadpercent"], ref_threads=r["threads"])
        print(f"{name}: reference {r['count']} (d padded to {ref_pad}, {rec['ref_s']} s)", flush=True)
    return rec


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", nargs="*", default=None)
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    args = ap.parse_args()
    doc = {"generator": "tests/golden/make_config_golden.py", "configs": {}}
    if os.path.exists(OUT):
        with open(OUT) as f:
            doc = json.load(f)
    for name in args.only or list(W.CONFIGS):
        doc["configs"][name] = run(name, args.threads)
        with open(OUT, "w") as f:
            json.dump(doc, f, indent=1, sort_keys=True)
            f.write("\n")


if __name__ == "__main__":
    main()
