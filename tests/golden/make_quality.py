"""Quality fixtures from GSAP's own GPU build (oracle/_ref/gsap_ref, which
oracle/build_ref.sh compiles from the reference tree) on the plain configs:

  * 20k-vertex DCSBM graphs, B=32, variants LL, LH, HL, HH, graph seeds 0-4;
  * the 200k-vertex HH graph of bench.py (graph seed 0), `--big-runs` runs.

For every run it records GSAP's final B, the MDL of its labels (computed
here by sbp_mdl in FP64, the same measure the tests use for our labels),
pairwise recall and precision against the planted labels, and its wall time.
GSAP seeds its RNG from clock64(), so each entry is one draw from its
run-to-run distribution.  Needs a GPU:

    python tests/golden/make_quality.py --out quality_ref.json [--big-runs 2]
    python tests/golden/make_quality.py --out quality_ref.json --only-big --append --big-runs 5
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from gsap_b200 import sbp  # noqa: E402

EXE = os.path.join(ROOT, "oracle", "_ref", "gsap_ref")
VARIANTS = ("LL", "LH", "HL", "HH")


def gsap_run(g, timeout):
    with tempfile.TemporaryDirectory() as td:
        gp, lp = os.path.join(td, "g.bin"), os.path.join(td, "l.bin")
        sbp.write_graph_bin(g, gp)
        t0 = time.perf_counter()
        p = subprocess.run([EXE, gp, "1", lp], capture_output=True, text=True, timeout=timeout)
        wall = (time.perf_counter() - t0) * 1000.0
        if p.returncode != 0:
            raise RuntimeError(f"gsap_ref exited {p.returncode}: {(p.stderr or p.stdout)[-300:]}")
        ms = json.loads(p.stdout.strip().splitlines()[-1])["ms"]
        lab = np.fromfile(lp, dtype=np.int32)
    return lab, ms, wall


def score(g, lab):
    B = int(lab.max()) + 1
    S, _ = sbp.mdl(g, lab, B)
    rec, prec, nmi = sbp.evaluate(g.true_partitions, lab)
    sizes = np.bincount(lab, minlength=B)
    return {"B": B, "S": S, "recall": rec, "precision": prec, "nmi": nmi,
            "largest_block": int(sizes.max()), "block0": int(sizes[0])}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default="quality_ref.json")
    ap.add_argument("--seeds", type=int, default=5)
    ap.add_argument("--big-runs", type=int, default=2)
    ap.add_argument("--timeout", type=float, default=600.0)
    ap.add_argument("--only-big", action="store_true", help="skip the 20k configs")
    ap.add_argument("--append", action="store_true",
                    help="add the new runs to the runs already in --out")
    a = ap.parse_args()
    out = {"generator": "sbp.dcsbm_variant(variant, N, B, seed); GSAP partition(g) via "
                        "oracle/_ref/gsap_ref; MDL and P/R computed on its final labels",
           "runs": []}
    if a.append and os.path.exists(a.out):
        out = json.load(open(a.out))
    big0 = sum(1 for r in out["runs"] if r["config"] == "200k")
    for v in (() if a.only_big else VARIANTS):
        for s in range(a.seeds):
            g = sbp.dcsbm_variant(v, 20000, 32, seed=s)
            lab, ms, wall = gsap_run(g, a.timeout)
            row = {"config": "20k", "variant": v, "graph_seed": s, "N": g.N, "E": g.E,
                   "ms": ms, "wall_ms": wall, **score(g, lab)}
            out["runs"].append(row)
            print(json.dumps(row), flush=True)
    g = sbp.dcsbm_variant("HH", 200000, 71, seed=0)
    for i in range(a.big_runs):
        lab, ms, wall = gsap_run(g, a.timeout)
        row = {"config": "200k", "variant": "HH", "graph_seed": 0, "run": big0 + i, "N": g.N,
               "E": g.E,
               "ms": ms, "wall_ms": wall, **score(g, lab)}
        out["runs"].append(row)
        print(json.dumps(row), flush=True)
    with open(a.out, "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
