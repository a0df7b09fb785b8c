"""End-to-end quality against GSAP's own GPU build.

tests/golden/quality_ref.json holds GSAP's results (final B, MDL of its
labels, pairwise recall and precision against the planted labels) on the
plain configs, written by tests/golden/make_quality.py on a B200.  Our
partitions of the same graphs must score an MDL within 1% of GSAP's and
pairwise recall / precision within 0.02 of GSAP's.

20k configs: partition seed = graph seed, five graph seeds, means against
means.  200k HH: five partition seeds of the benchmark graph against every
GSAP run on record (at least five; GSAP seeds its RNG from clock64(), so
each run is a fresh draw).  There GSAP's recall has a heavy tail (one draw
in eight ended with one block holding most vertices, recall 0.61, against
0.011-0.028 for the others), so the bar compares our mean with GSAP's
median of each score; the MDL bar also holds against GSAP's mean."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "quality_ref.json")


def _ref(config, variant):
    runs = json.load(open(FIX))["runs"]
    return [r for r in runs if r["config"] == config and r["variant"] == variant]


def _ours(sbp, variant, N, B, graph_seeds, part_seeds):
    out = []
    for gs, ps in zip(graph_seeds, part_seeds):
        g = sbp.dcsbm_variant(variant, N, B, seed=gs)
        rep = sbp.partition(g, seed=ps)
        rec, prec, _ = sbp.evaluate(g.true_partitions, g.partitions)
        out.append((rep["S"], rec, prec))
    return np.array(out)


def _check(ours, ref):
    S, rec, prec = ours.mean(axis=0)
    S_ref = np.mean([r["S"] for r in ref])
    rec_ref = np.mean([r["recall"] for r in ref])
    prec_ref = np.mean([r["precision"] for r in ref])
    assert abs(S - S_ref) <= 0.01 * S_ref, (S, S_ref)
    assert abs(rec - rec_ref) <= 0.02, (rec, rec_ref)
    assert abs(prec - prec_ref) <= 0.02, (prec, prec_ref)


@pytest.mark.parametrize("variant", ["LL", "LH", "HL", "HH"])
def test_20k_quality_matches_gsap(sbp, variant):
    ref = _ref("20k", variant)
    assert len(ref) == 5
    seeds = [r["graph_seed"] for r in ref]
    _check(_ours(sbp, variant, 20000, 32, seeds, seeds), ref)


def test_200k_quality_matches_gsap(sbp):
    ref = _ref("200k", "HH")
    assert len(ref) >= 5
    ours = _ours(sbp, "HH", 200000, 71, [0] * 5, [0, 1, 2, 3, 4])
    S, rec, prec = ours.mean(axis=0)
    med = {k: float(np.median([r[k] for r in ref])) for k in ("S", "recall", "precision")}
    mean = {k: float(np.mean([r[k] for r in ref])) for k in ("S", "recall", "precision")}
    assert abs(S - med["S"]) <= 0.01 * med["S"], (S, med, mean)
    assert abs(rec - med["recall"]) <= 0.02, (rec, med, mean)
    assert abs(prec - med["precision"]) <= 0.02, (prec, med, mean)
    assert abs(S - mean["S"]) <= 0.01 * mean["S"], (S, mean)
