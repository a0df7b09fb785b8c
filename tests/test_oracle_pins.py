"""Pins the CPU oracle to the reference itself.

The golden files in tests/golden were produced by GSAP's own code
(tests/golden/make_golden.py): its kernels (kernels.hpp, FP32 with log2f),
its evaluator (evaluate.hpp) and its loader (load.hpp).  The oracle computes
in FP64, so dS agrees to FP32 rounding: |oracle - ref| <= 2e-6 * (sum of the
magnitudes of the terms), a bound that covers the FP32 accumulation of
terms of size up to ~1e5.
"""
import glob
import json
import os

import numpy as np
import pytest

import refkernels as rk

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
KERN = sorted(glob.glob(os.path.join(GOLD, "refkern_*.npz")))


def _close32(got, ref, scale):
    with np.errstate(invalid="ignore"):
        return (got == ref) | (np.abs(got - ref) <= 2e-6 * np.maximum(scale, 1.0))


def _graph(sbp, z):
    return sbp.Graph.from_edges(int(z["N"]), z["src"], z["dst"], z["w"])


@pytest.mark.parametrize("path", KERN, ids=[os.path.basename(p) for p in KERN])
def test_nodal_terms_match_reference_kernels(sbp, orc, path):
    z = np.load(path)
    g = _graph(sbp, z)
    B, BS, itr = int(z["B"]), int(z["BS"]), int(z["itr"])
    part, props = z["part"], z["props"]
    verts = np.arange(itr * BS, (itr + 1) * BS, dtype=np.int32)
    r, s = part[verts], props[verts]
    dso = z["dS_out"].astype(np.float64)
    t = z["terms"].astype(np.float64)
    ref = dso[r] + dso[s] + t[0] + t[1] - t[2] - t[3] - t[4] - t[5]
    ref[r == s] = 0.0
    scale = np.abs(dso[r]) + np.abs(dso[s]) + np.abs(t).sum(axis=0)
    got, q3 = orc.nodal_delta(g, part, B, verts, s)
    # moves whose in-list runs past block s's in-row read an out-of-row
    # weight in the reference (kernels.hpp:1348-1358); the oracle uses the
    # list's own weight there
    ok = _close32(got, ref, scale)
    assert ok[~q3].all(), np.flatnonzero(~ok & ~q3)[:5]
    # the accept decisions agree wherever dS is not within FP32 noise of 0
    acc_ref = z["accepted"] < 0
    clear = (np.abs(ref) > 1e-3 * np.maximum(scale, 1.0)) & ~q3
    assert np.array_equal((got < 0)[clear], acc_ref[clear])


@pytest.mark.parametrize("path", KERN, ids=[os.path.basename(p) for p in KERN])
def test_merge_dS_matches_reference_kernels(sbp, orc, path):
    z = np.load(path)
    g = _graph(sbp, z)
    B = int(z["B"])
    got, _, _ = orc.merge_delta(g, z["part"], B, z["merge_props"])
    ref = z["merge_dS"].astype(np.float64)
    # every term of a merge is w (log2 w - log2 d - log2 d') with |.| below
    # w * 2 log2(E); the four rows involved carry the weight of both blocks'
    # degrees, counted for the old and the merged rows
    bm = orc.build_blockmodel(g, z["part"], B)
    r = np.repeat(np.arange(B), 10)
    s = z["merge_props"]
    deg = (bm["d_out"].astype(np.float64) + bm["d_in"])
    scale = 4.0 * np.log2(g.E) * (deg[r] + deg[s]) + 1.0
    assert _close32(got, ref, scale).all()


@pytest.mark.parametrize("path", KERN, ids=[os.path.basename(p) for p in KERN])
def test_mdl_matches_reference(sbp, orc, path):
    z = np.load(path)
    g = _graph(sbp, z)
    S, dataS = orc.mdl(g, z["part"], int(z["B"]))
    assert abs(dataS - float(z["data_S"])) <= 1e-5 * abs(float(z["data_S"]))
    assert abs(S - float(z["S"])) <= 1e-5 * abs(float(z["S"]))


@pytest.mark.skipif(not rk.available, reason="reference kernels not built here")
@pytest.mark.parametrize("B", [3, 40, 400, 1000])
def test_live_nodal_terms_sparse_rows(sbp, orc, B):
    """Live run of the reference kernels on sparse blockmodels, where the
    split-term and missing-column paths of the new-row kernels fire."""
    g = sbp.dcsbm_variant("HH", 1000, 11, seed=B)
    rng = np.random.default_rng(B)
    part = rng.integers(0, B, g.N).astype(np.int32)
    part[:B] = np.arange(B, dtype=np.int32)
    bm = orc.build_blockmodel(g, part, B)
    BS = g.N // 4
    for itr in range(4):
        props = rng.integers(0, B, g.N).astype(np.int32)
        dso, terms, acc, _ = rk.nodal_batch(g, part, B, bm, props, BS, itr)
        verts = np.arange(itr * BS, (itr + 1) * BS, dtype=np.int32)
        r, s = part[verts], props[verts]
        t = terms.astype(np.float64)
        ref = dso[r].astype(np.float64) + dso[s] + t[0] + t[1] - t[2] - t[3] - t[4] - t[5]
        ref[r == s] = 0.0
        scale = np.abs(dso[r]) + np.abs(dso[s]) + np.abs(t).sum(axis=0)
        got, q3 = orc.nodal_delta(g, part, B, verts, s)
        ok = _close32(got, ref, scale)
        assert ok[~q3].all()


@pytest.mark.skipif(not rk.available, reason="reference kernels not built here")
def test_live_accepted_prob(sbp, orc):
    g = sbp.dcsbm_variant("LL", 1000, 11, seed=0)
    part = g.true_partitions
    bm = orc.build_blockmodel(g, part, 11)
    ap = rk.accepted_prob(11, bm)
    d = bm["d_out"].astype(np.float64) + bm["d_in"]
    np.testing.assert_allclose(ap, 11.0 / (d + 11.0), rtol=1e-6)


def _pairs_numpy(t, gv):
    tab = np.zeros((t.max() + 1, gv.max() + 1), np.int64)
    np.add.at(tab, (t, gv), 1)
    c2 = lambda x: (x * (x - 1) // 2).sum()
    same = c2(tab)
    pj = tab / tab.sum()
    pr, pc = pj.sum(1), pj.sum(0)
    nz = pj > 0
    mi = (pj[nz] * np.log(pj[nz] / np.outer(pr, pc)[nz])).sum()
    h = lambda q: -(q[q > 0] * np.log(q[q > 0])).sum()
    return same / c2(tab.sum(1)), same / c2(tab.sum(0)), 2 * mi / (h(pr) + h(pc))


def test_evaluator_matches_reference(sbp, orc):
    gold = json.load(open(os.path.join(GOLD, "evaluate.json")))
    z = np.load(os.path.join(GOLD, "evaluate_inputs.npz"))
    for key, want in gold.items():
        t, gv = z[key + "_truth"], z[key + "_given"]
        for got in (orc.evaluate(t, gv), sbp.evaluate(t, gv)):
            np.testing.assert_allclose(got, _pairs_numpy(t, gv), rtol=1e-12)
            if t.max() != gv.max():
                continue  # reference table corrupted by its column fill-in
            r, p, nmi = got
            # the reference prints 6 significant digits of float arithmetic
            assert abs(r - want["recall"]) <= 2e-6 + 1e-5 * want["recall"]
            assert abs(p - want["precision"]) <= 2e-6 + 1e-5 * want["precision"]
            assert abs(nmi - want["nmi"]) <= 1e-4


def test_philox_known_answers(orc):
    # Random123 philox4x32-10 known-answer vectors
    kat = [([0, 0, 0, 0], [0, 0], [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]),
           ([0xffffffff] * 4, [0xffffffff] * 2, [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]),
           ([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0],
            [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1])]
    for ctr, key, want in kat:
        assert list(orc.philox(ctr, key)) == want
