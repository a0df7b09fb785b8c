"""Blockmodels pinned to GSAP's own builder, calculate_new_csr
(GSAP/partition.hpp:707-849): tests/golden/gsap_csr.json holds the SHA-256
of every array GSAP built on seeded graphs and partitions
(tests/golden/make_csr_golden.py, run on a B200).  The oracle's builder
(CPU) and the partitioner's (GPU, through the C ABI) must give the same
bytes: row pointers without the end sentinel, ascending columns, counts and
row degrees of the out and the in CSR."""
import hashlib
import json
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
FIX = os.path.join(HERE, "golden", "gsap_csr.json")

pytestmark = pytest.mark.skipif(not os.path.exists(FIX), reason="GSAP builder fixture missing")


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _ours(bm):
    return {"out_ptr": bm["optr"][:-1], "out_col": bm["ocol"], "out_cnt": bm["ocnt"],
            "out_deg": bm["d_out"], "in_ptr": bm["iptr"][:-1], "in_col": bm["icol"],
            "in_cnt": bm["icnt"], "in_deg": bm["d_in"]}


def _check(build, name):
    import make_csr_golden as m
    want = json.load(open(FIX))["graphs"][name]
    g, cases = m.cases_for(name)
    assert (g.N, g.E) == (want["N"], want["E"])
    assert [c[0] for c in cases] == [w["case"] for w in want["cases"]]
    for (case, p, B), w in zip(cases, want["cases"]):
        assert B == w["B"], case
        got = _ours(build(g, p, B))
        assert got["out_col"].size == w["nnz_out"] and got["in_col"].size == w["nnz_in"], case
        for k in m.KEYS:
            assert _sha(got[k]) == w[k], (case, k)


@pytest.mark.parametrize("name", ["LL1k", "HH1k", "HH20k"])
def test_oracle_builder_matches_gsap(orc, name):
    _check(orc.build_blockmodel, name)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["LL1k", "HH1k", "HH20k"])
def test_gpu_builder_matches_gsap(sbp, orc, name):
    def build(g, p, B):
        from gsap_b200 import sbp as s
        gg = s.Graph(N=g.N, E=g.E, out_ptr=g.out_ptr, out_idx=g.out_idx, out_w=g.out_w,
                     in_ptr=g.in_ptr, in_idx=g.in_idx, in_w=g.in_w, deg_out=g.deg_out,
                     deg_in=g.deg_in)
        return s.build_blockmodel(gg, p, B)
    _check(build, name)
