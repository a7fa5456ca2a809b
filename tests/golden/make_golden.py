"""Regenerates the golden fixtures in this directory.

Sources (read only here, never at test time):
  * the reference's published H100 results,
    results/{zeta,random}/summary/all_results.json -- the f64 programs' first
    100 per-trajectory rows for every CMF x mode, and the df64 / RNS summary
    counters;
  * the reference's own kernel bodies compiled for the host (oracle/_ref,
    built by `make -C oracle ref`) -- RNS residue traces and df64 / RNS
    result rows, which the reference never publishes.

Usage: python tests/golden/make_golden.py [REFERENCE_ROOT]
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def published(ref_root):
    rows, summaries = [], []
    for kind, zeta in (("zeta", True), ("random", False)):
        path = os.path.join(ref_root, "results", kind, "summary", "all_results.json")
        with open(path) as f:
            data = json.load(f)
        for r in data:
            p, q = (int(x) for x in r["cmf"].split("F"))
            key = {"variant": r["variant"], "cmf": r["cmf"], "p": p, "q": q, "z": r["z"],
                   "zeta": zeta, "mode": r["mode"], "N": r["N"], "h": r["h"], "n_traj": r["n_traj"],
                   "rank": r["rank"]}
            summaries.append(dict(key, n_valid=r["n_valid"], n_with_limits=r["n_with_limits"],
                                  avg_delta=r["avg_delta"]))
            if r.get("results"):
                rows.append(dict(key, results=r["results"]))
    with open(os.path.join(HERE, "published_f64_rows.json"), "w") as f:
        json.dump(rows, f, separators=(",", ":"))
    with open(os.path.join(HERE, "published_summaries.json"), "w") as f:
        json.dump(summaries, f, indent=1)


def reference_runs():
    import oracle
    if not oracle.have_ref("rns"):
        raise SystemExit("oracle/_ref is not built: run `make -C oracle ref` first")
    cases = []
    # RNS residue traces on trajectories the walk keeps valid, for both
    # roundings of the column polynomial.
    picks = [(3, 2, 0.5, [3, 5, 7, 4, 6], [1, 1, 1, 1, 1]),
             (3, 2, 0.5, [2, 9, 4, 7, 3], [1, 0, 1, 0, 0]),
             (4, 3, 0.5, [5, 3, 8, 2, 6, 9, 4], [1, 0, 0, 1, 0, 0, 0]),
             (5, 4, 1.0, [1, 1, 1, 1, 1, 2, 2, 2, 2], [1, 0, 0, 0, 0, 0, 0, 0, 0]),
             (6, 5, 1.0, [1] * 6 + [2] * 5, [0, 0, 1, 3, 0, 1, 0, 0, 0, 0, 0]),
             (8, 7, 0.5, [3, 4, 5, 6, 7, 8, 9, 10, 4, 5, 6, 7, 8, 9, 10], [1] + [0] * 14)]
    for p, q, z, start, d in picks:
        rank = max(p, q + 1) - (1 if (z == 1.0 and p == q + 1) else 0)
        for fused in (False, True):
            for K, steps in ((8, 150), (13, 250), (64, 120)):
                ok, res, ls = oracle.ref_rns_trace(p, q, z, 300, 50, d, start, K, steps, rank, fused=fused)
                cases.append({"kind": "rns_trace", "p": p, "q": q, "z": z, "start": start, "dir": d,
                              "N": 300, "h": 50, "n_primes": K, "steps": steps, "rank": rank,
                              "fused": fused, "ok": ok, "log_scale": ls,
                              "residues": res.reshape(-1).tolist()})
    # Whole-program rows of every variant on the reference's own inputs.
    for p, q, z, zeta, mode in ((3, 2, 0.5, False, 0), (6, 5, 1.0, True, 0), (4, 3, 0.5, False, 0)):
        recs = oracle.ref_make_inputs(p, q, 400, mode, zeta)[:24]
        for variant, N, h in (("f64", 400, 40), ("df64", 400, 40), ("rns", 200, 20)):
            out = oracle.ref_walk(variant, p, q, z, N, h, recs, n_primes=8, fused=False)
            rows = []
            for r in out:
                rows.append({k: (None if not np.isfinite(r[k]) else float(r[k]))
                             for k in ("limit", "delta", "p", "q", "precision", "log_scale")})
                rows[-1]["valid"] = int(r["valid"])
                rows[-1]["n_limits"] = int(r["n_limits"])
                if not r["valid"]:
                    rows[-1]["p"] = rows[-1]["q"] = None  # never written by the reference
            cases.append({"kind": "rows", "variant": variant, "p": p, "q": q, "z": z, "zeta": zeta,
                          "mode": mode, "N": N, "h": h, "n": 24, "rows": rows})
    with open(os.path.join(HERE, "reference_host_runs.json"), "w") as f:
        json.dump(cases, f, separators=(",", ":"))


if __name__ == "__main__":
    ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CMFW_REF_ROOT")
    if not ref_root:
        sys.exit("usage: make_golden.py <reference checkout> (or set CMFW_REF_ROOT)")
    published(ref_root)
    reference_runs()
    print("golden fixtures written to", HERE)
