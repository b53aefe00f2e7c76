"""Generates tests/golden/golden_counts.json.

Each case is a seeded synthetic point set (regenerated at test time from
``hilbertjoin_b200.workloads``; no point data is stored). For every case this
script records:

* ``ref_count``: the count of the hilbertJoin reference built from its own
  sources (``oracle/build_ref.sh``), called through its library entry points
  ``test_ego_loop3_macro`` / ``test_ego_loop3_noself`` with the
  dimension-reordering pre-step skipped (see ``oracle/ref_driver.cpp``);
* ``oracle_count``: the brute-force FP64 count of ``oracle/hj_oracle.c``;
* ``ref_valid``: whether the case lies in the domain where the reference is
  expected to be exact (d >= 8, continuous data, n % 8 == 0, nB <= nA). Outside
  it the reference's value is recorded to document how it differs.

Run from the repository root:  python tests/golden/make_golden.py
It needs the reference sources (to build ``oracle/_ref``) and takes about a
minute on 8 cores.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from hilbertjoin_b200 import workloads as W  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden_counts.json")


def make(spec: dict):
    g = spec["gen"]
    if g == "uniform":
        x = W.uniform(spec["n"], spec["d"], spec["seed"])
    elif g == "uniform_f32":
        x = W.uniform(spec["n"], spec["d"], spec["seed"], dtype=np.float32).astype(np.float64)
    elif g == "gmm":
        x = W.gmm(spec["n"], spec["d"], spec["seed"])
    elif g == "lattice":
        x = W.lattice(spec["n"], spec["d"], spec["seed"], levels=spec.get("levels", 10))
    else:
        raise ValueError(g)
    pad = spec.get("pad_to", spec["d"])
    if pad > spec["d"]:
        x = np.concatenate([x, np.zeros((x.shape[0], pad - spec["d"]))], axis=1)
    return x


def cases():
    out = []
    # self-joins, uniform, eps for ~20 neighbours per point
    for d in (8, 16, 32, 64):
        out.append(dict(name=f"self_uniform_d{d}", kind="self", gen="uniform", n=4000, d=d, seed=100 + d,
                        nbrs=20))
    # the README example shape at reduced n: eps = 0.2 at d = 64 has no pairs
    out.append(dict(name="self_uniform_d64_eps0.2", kind="self", gen="uniform", n=8000, d=64, seed=1, eps=0.2))
    # FP32-rounded dense regime (config-3 shape at reduced n, ~32 neighbours)
    out.append(dict(name="self_uniform_f32_d64_dense", kind="self", gen="uniform_f32", n=4000, d=64, seed=22,
                    nbrs=32, nbrs_n=1_000_000))
    # clustered, config-4 shape at reduced n; d=28 zero-padded to 32 is the reference's CLI workaround
    out.append(dict(name="self_gmm_d28", kind="self", gen="gmm", n=6000, d=28, seed=44, nbrs=100))
    out.append(dict(name="self_gmm_d28_pad32", kind="self", gen="gmm", n=6000, d=28, seed=44, nbrs=100,
                    pad_to=32))
    # two-set joins (A and B from independent seeds), eps for ~20 partners
    for d in (8, 20, 24, 64):
        out.append(dict(name=f"join_uniform_d{d}", kind="join", gen="uniform", n=4000, m=4000, d=d, seed=200 + d,
                        seed_b=300 + d, nbrs=20))
    out.append(dict(name="join_uniform_d20_eps0.2", kind="join", gen="uniform", n=4000, m=3200, d=20, seed=1,
                    seed_b=2, eps=0.2))
    # outside the reference's valid domain: recorded to document the differences
    out.append(dict(name="self_lattice_d8_ties", kind="self", gen="lattice", n=4000, d=8, seed=7, levels=3,
                    eps=0.1))
    out.append(dict(name="self_uniform_d4", kind="self", gen="uniform", n=4000, d=4, seed=104, nbrs=20))
    out.append(dict(name="self_uniform_tail_n4005", kind="self", gen="uniform", n=4005, d=16, seed=116, nbrs=20))
    return out


def main():
    res = []
    for c in cases():
        x = make(c)
        if "eps" not in c:
            if c["kind"] == "self":
                c["eps"] = W.calibrate_eps(x, c.get("nbrs_n", c["n"]), c["nbrs"])
            else:
                b = make(dict(c, seed=c["seed_b"], n=c["m"]))
                c["eps"] = W.calibrate_eps_join(x, b, c["m"], c["nbrs"])
        eps = c["eps"]
        if c["kind"] == "self":
            r = oracle.ref_self_count(x, eps, stripes=14)
            o = oracle.self_count_brute(x, eps)
            o_tail = oracle.self_count_ego(x, eps, 3, tail_drop=True)[0]
            valid = c["d"] >= 8 and c["gen"] != "lattice" and c["n"] % 8 == 0
        else:
            b = make(dict(c, seed=c["seed_b"], n=c["m"]))
            r = oracle.ref_join_count(x, b, eps)
            o = oracle.join_count_brute(x, b, eps)
            o_tail = oracle.join_count_ego(x, b, eps, 2, tail_drop=True)[0]
            valid = c["d"] >= 8 and c["n"] % 8 == 0 and c["m"] % 8 == 0 and c["m"] <= c["n"]
        c.update(ref_count=int(r["count"]), ref_loadpercent=r["loadpercent"], oracle_count=o,
                 oracle_count_tail_drop=o_tail, ref_valid=bool(valid))
        print(f"{c['name']:32s} eps={eps:<12g} ref={c['ref_count']:<9d} oracle={o:<9d} "
              f"tail_drop={o_tail:<9d} valid={valid}", flush=True)
        res.append(c)
    with open(OUT, "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "cases": res}, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
