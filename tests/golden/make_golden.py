"""Generates the golden fixtures of this directory from the reference itself.

Needs the reference tree (REF, else the tree oracle/build_ref.sh used) and the checkers
that oracle/build_ref.sh builds from it into oracle/_ref/:

  loader.json       GSAP/load.hpp on the eight bundled 1k/5k GraphChallenge
                    graphs: N, E and a SHA-256 of every array it fills
  evaluate.json     GSAP/evaluate/evaluate.hpp on seeded (truth, given) pairs
                    stored in evaluate_inputs.npz
  refkern_*.npz     GSAP/kernels.hpp (nodal dS terms, merge dS, MDL) run on
                    seeded inputs stored in the same file

    python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

REF = os.environ.get("REF", "")
if not REF and os.path.exists(os.path.join(ROOT, "oracle", "_ref", "ref_root")):
    REF = open(os.path.join(ROOT, "oracle", "_ref", "ref_root")).read().strip()
REF_HOST = os.path.join(ROOT, "oracle", "_ref", "ref_host")
CATS = ("LL", "LH", "HL", "HH")
SIZES = ("1k", "5k")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def read_ref_graph(path):
    with open(path, "rb") as f:
        N, E = np.frombuffer(f.read(8), np.int32)
        out = {}
        for name, dt in (("out_ptr", np.int32), ("out_idx", np.int32), ("out_w", np.uint32),
                         ("in_ptr", np.int32), ("in_idx", np.int32), ("in_w", np.uint32),
                         ("deg_out", np.uint32), ("deg_in", np.uint32), ("truth", np.int32)):
            n = int(np.frombuffer(f.read(8), np.int64)[0])
            out[name] = np.frombuffer(f.read(4 * n), dt).copy()
    return int(N), int(E), out


def loader_goldens():
    res = {}
    with tempfile.TemporaryDirectory() as td:
        for c in CATS:
            for s in SIZES:
                p = os.path.join(td, f"{c}{s}.bin")
                subprocess.run([REF_HOST, "load", c, s, p], cwd=os.path.join(REF, "GSAP"),
                               check=True)
                N, E, arr = read_ref_graph(p)
                res[f"{c}-{s}"] = {"N": N, "E": E, **{k: sha(v) for k, v in arr.items()}}
    return res


def evaluate_goldens():
    from gsap_b200 import sbp
    rng = np.random.default_rng(2024)
    inputs, outs = {}, {}
    k = 0
    for N, B, variant in ((1000, 11, "LL"), (1000, 11, "HH"), (5000, 19, "LH")):
        truth = sbp.dcsbm_variant(variant, N, B, seed=k).true_partitions
        # equal block counts, where evaluate.hpp's table is a column
        # permutation, plus two unequal ones (its column fill-in at
        # evaluate.hpp:93-108 drops and repeats columns there)
        for noise, Bg in ((0.0, B), (0.1, B), (0.3, B), (0.6, B), (1.0, B), (0.4, B + 5),
                          (0.2, 2 * B)):
            given = truth.copy() % Bg
            flip = rng.random(N) < noise
            given[flip] = rng.integers(0, Bg, flip.sum())
            # labels must be 0..max without gaps above, as GSAP's partitions are
            given = np.unique(given, return_inverse=True)[1].astype(np.int32)
            key = f"case{k}"
            inputs[key + "_truth"] = truth.astype(np.int32)
            inputs[key + "_given"] = given
            with tempfile.TemporaryDirectory() as td:
                a, b = os.path.join(td, "t.bin"), os.path.join(td, "g.bin")
                truth.astype(np.int32).tofile(a)
                given.tofile(b)
                out = subprocess.run([REF_HOST, "eval", str(N), a, b], capture_output=True,
                                     text=True, check=True).stdout
            vals = {}
            for line in out.splitlines():
                name, _, v = line.partition(":")
                vals[name.strip()] = float(v)
            outs[key] = {"recall": vals["Pairwise Recall"],
                         "precision": vals["Pairwise Precision"],
                         "nmi": vals["Normalized Mutual Information(NMI)"]}
            k += 1
    np.savez_compressed(os.path.join(HERE, "evaluate_inputs.npz"), **inputs)
    return outs


def kernel_goldens():
    import refkernels as rk
    from gsap_b200 import sbp
    from oracle import oracle as orc
    cases = [("HH1k_B20", sbp.dcsbm_variant("HH", 1000, 11, seed=3), 20, 0),
             ("LL1k_B300", sbp.dcsbm_variant("LL", 1000, 11, seed=4), 300, 1),
             ("HL1k_identity", sbp.dcsbm_variant("HL", 1000, 11, seed=5), 1000, 2)]
    for name, g, B, seed in cases:
        rng = np.random.default_rng(seed)
        part = rng.integers(0, B, g.N).astype(np.int32)
        part[:B] = np.arange(B, dtype=np.int32)
        bm = orc.build_blockmodel(g, part, B)
        BS = g.N // 4
        itr = 1
        props = rng.integers(0, B, g.N).astype(np.int32)
        src, dst, w = g.edges()
        pick = rng.integers(0, g.E, g.N)
        props = np.where(rng.random(g.N) < 0.6, part[dst[pick]], props).astype(np.int32)
        dso, terms, acc, _ = rk.nodal_batch(g, part, B, bm, props, BS, itr)
        mprops = orc.merge_proposals(g, part, B, seed=seed, seq=3)
        mdS = rk.merge_delta(B, bm, mprops)
        S, dataS = rk.mdl(B, g.N, g.E, bm)
        aprob = rk.accepted_prob(B, bm)
        np.savez_compressed(
            os.path.join(HERE, f"refkern_{name}.npz"), N=g.N, src=src, dst=dst, w=w, part=part,
            B=B, BS=BS, itr=itr, props=props, dS_out=dso, terms=terms, accepted=acc,
            merge_props=mprops, merge_dS=mdS, S=S, data_S=dataS, accepted_prob=aprob)


if __name__ == "__main__":
    if not (os.path.isdir(os.path.join(REF, "GSAP")) and os.path.exists(REF_HOST)):
        sys.exit("needs the reference tree and oracle/_ref (run oracle/build_ref.sh)")
    with open(os.path.join(HERE, "loader.json"), "w") as f:
        json.dump(loader_goldens(), f, indent=1, sort_keys=True)
    with open(os.path.join(HERE, "evaluate.json"), "w") as f:
        json.dump(evaluate_goldens(), f, indent=1, sort_keys=True)
    kernel_goldens()
    print("goldens written to", HERE)
