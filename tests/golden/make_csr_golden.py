"""Blockmodel fixtures from GSAP's own builder: calculate_new_csr
(GSAP/partition.hpp:707-849) run by oracle/_ref/gsap_csr (built from the
reference tree by oracle/build_ref.sh) on seeded graphs and partitions.
Records, per case, the block count, the nonzero counts and the SHA-256 of
every array GSAP builds (row pointers without the end sentinel, columns,
counts, row degrees; out and in).  Graphs come from the oracle's generator,
with unit weights (GSAP's builder assumes them, Q13).  Needs a GPU:

    python tests/golden/make_csr_golden.py --out gsap_csr.json
"""
import argparse
import hashlib
import json
import os
import struct
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as orc  # noqa: E402

EXE = os.path.join(ROOT, "oracle", "_ref", "gsap_csr")
KEYS = ("out_ptr", "out_col", "out_cnt", "out_deg", "in_ptr", "in_col", "in_cnt", "in_deg")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def cases_for(name):
    """(graph, [(case name, labels, B)]) of one fixture graph."""
    v, N, B0, seed = {"LL1k": ("LL", 1000, 11, 0), "HH1k": ("HH", 1000, 11, 1),
                      "HH20k": ("HH", 20000, 32, 0)}[name]
    g = orc.dcsbm_variant(v, N, B0, seed=seed)
    rng = np.random.default_rng(seed + 17)
    out = [("identity", np.arange(N, dtype=np.int32), N),
           ("planted", g.true_partitions.astype(np.int32), B0)]
    for B in (7, 40, N // 10):
        p = rng.integers(0, B, N).astype(np.int32)
        p[:B] = np.arange(B, dtype=np.int32)
        out.append((f"random{B}", p, B))
    k = int(np.float32(N) * np.float32(0.35))
    merged, nb, _, _ = orc.merge_step(g, np.arange(N, dtype=np.int32), N, k, 0, 0, ref_grid=1)
    out.append(("first-merge", merged, nb))
    return g, out


def run(g, cases):
    with tempfile.TemporaryDirectory() as td:
        gp, cp, op = (os.path.join(td, x) for x in ("g.bin", "c.bin", "o.bin"))
        orc.write_graph_bin(g, gp)
        with open(cp, "wb") as f:
            f.write(struct.pack("<i", len(cases)))
            for _, p, B in cases:
                f.write(struct.pack("<i", B))
                f.write(np.ascontiguousarray(p, np.int32).tobytes())
        r = subprocess.run([EXE, gp, cp, op], capture_output=True, text=True, timeout=900)
        if r.returncode != 0:
            raise RuntimeError(f"gsap_csr exited {r.returncode}: {r.stderr[-400:]}")
        raw = np.fromfile(op, dtype=np.int32)
    out, at = [], 0
    for name, _, B in cases:
        b, no, ni = raw[at:at + 3]
        at += 3
        assert b == B
        arrs = {}
        for key, n in zip(KEYS, (B, no, no, B, B, ni, ni, B)):
            arrs[key] = raw[at:at + n]
            at += n
        row = {"case": name, "B": int(B), "nnz_out": int(no), "nnz_in": int(ni)}
        row.update({k: sha(arrs[k]) for k in KEYS})
        out.append(row)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default="gsap_csr.json")
    a = ap.parse_args()
    res = {"builder": "GSAP calculate_new_csr (partition.hpp:707-849) via oracle/_ref/gsap_csr",
           "graphs": {}}
    for name in ("LL1k", "HH1k", "HH20k"):
        g, cases = cases_for(name)
        res["graphs"][name] = {"N": g.N, "E": g.E, "cases": run(g, cases)}
        print(name, "done", flush=True)
    with open(a.out, "w") as f:
        json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
