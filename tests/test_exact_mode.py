"""Exact-MDL and Metropolis-Hastings scoring on the GPU against the oracle.

Bars: dS within 1e-9 relative (|gpu - oracle| <= 1e-9 * max(|oracle|, 1
bit)); log Hastings ratios within 1e-10; proposals, accepted moves and
labels bit-exact.  The oracle's exact mode is itself pinned to brute-force
MDL differences (test_exact_oracle.py).
"""
import numpy as np
import pytest

import graphs
from test_exact_oracle import _self_loop_graph

pytestmark = pytest.mark.gpu

REL = 1e-9
LOGH_TOL = 1e-10


def close(a, b, rel=REL):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return (a == b) | (np.abs(a - b) <= rel * np.maximum(np.abs(b), 1.0))


def _graphs(sbp):
    return {"LL1k": graphs.dcsbm("LL", 1000, 11, 0),
            "HH1k": graphs.dcsbm("HH", 1000, 11, 1),
            "weighted": graphs.weighted_graph(),
            "self_loops": _self_loop_graph(sbp, N=800)}


@pytest.fixture(scope="module")
def gs(sbp):
    return _graphs(sbp)


def _partition(g, B, seed):
    p = np.random.default_rng(seed).integers(0, B, g.N).astype(np.int32)
    p[:B] = np.arange(B, dtype=np.int32)
    return p


FORMS = [("dense", "4096"), ("csr", "0")]
GRAPHS = ["LL1k", "HH1k", "weighted", "self_loops"]


@pytest.mark.parametrize("form,dmax", FORMS, ids=[f[0] for f in FORMS])
@pytest.mark.parametrize("name", GRAPHS)
@pytest.mark.parametrize("B", [5, 40, 300])
def test_exact_nodal_dS_and_hastings(sbp, orc, gs, name, B, form, dmax, monkeypatch):
    monkeypatch.setenv("SBP_DENSE_MAX", dmax)
    g = gs[name]
    p = _partition(g, B, B)
    rng = np.random.default_rng(B + 1)
    verts = np.arange(g.N, dtype=np.int32)
    props = rng.integers(0, B, g.N).astype(np.int32)
    got, lh = sbp.delta_mdl_nodal_mode(g, p, B, verts, props, exact=1)
    want, lh_o = orc.nodal_delta_exact(g, p, B, verts, props)
    ok = close(got, want)
    assert ok.all(), (np.flatnonzero(~ok)[:5], got[~ok][:5], want[~ok][:5])
    assert (np.abs(lh - lh_o) <= LOGH_TOL).all()


@pytest.mark.parametrize("name", GRAPHS)
def test_general_kernel_with_gsap_terms(sbp, orc, gs, name):
    # exact = 0 in the general-mode kernel: GSAP's dS, plus the Hastings ratio
    g = gs[name]
    B = 40
    p = _partition(g, B, 3)
    verts = np.arange(g.N, dtype=np.int32)
    props = np.random.default_rng(4).integers(0, B, g.N).astype(np.int32)
    got, lh = sbp.delta_mdl_nodal_mode(g, p, B, verts, props, exact=0)
    want, _ = orc.nodal_delta(g, p, B, verts, props)
    _, lh_o = orc.nodal_delta_exact(g, p, B, verts, props)
    with np.errstate(invalid="ignore"):
        assert close(got, want).all()
    assert (np.abs(lh - lh_o) <= LOGH_TOL).all()


@pytest.mark.parametrize("which", ["identity", "planted", "random100"])
def test_exact_heavy_vertices(sbp, orc, which):
    # vertex 0: ~9000 in-entries (hashed passes), vertex 1: ~1000 (CTA sort)
    g = graphs.hub_graph()
    if which == "identity":
        p, B = np.arange(g.N, dtype=np.int32), g.N
    elif which == "planted":
        p, B = g.true_partitions, int(g.true_partitions.max()) + 1
    else:
        B = 100
        p = _partition(g, B, 3)
    rng = np.random.default_rng(7)
    verts = np.concatenate([[0, 1], rng.integers(2, g.N, 3000)]).astype(np.int32)
    props = rng.integers(0, B, verts.size).astype(np.int32)
    got, lh = sbp.delta_mdl_nodal_mode(g, p, B, verts, props, exact=1)
    want, lh_o = orc.nodal_delta_exact(g, p, B, verts, props)
    ok = close(got, want)
    assert ok.all(), (np.flatnonzero(~ok)[:5], got[~ok][:5], want[~ok][:5])
    assert (np.abs(lh - lh_o) <= LOGH_TOL).all()


def test_exact_moves_are_mdl_differences(sbp, gs):
    # the GPU's exact dS against two full MDL evaluations of its own
    g = gs["self_loops"]
    B = 12
    p = _partition(g, B, 9)
    verts = np.arange(0, g.N, 7, dtype=np.int32)
    props = np.random.default_rng(2).integers(0, B, verts.size).astype(np.int32)
    got, _ = sbp.delta_mdl_nodal_mode(g, p, B, verts, props, exact=1, hastings=False)
    S0, _ = sbp.mdl(g, p, B)
    for i, v in enumerate(verts):
        q = p.copy()
        q[v] = props[i]
        S1, _ = sbp.mdl(g, q, B)
        assert abs(got[i] - (S1 - S0)) <= 1e-9 * abs(S0)


@pytest.mark.parametrize("name", GRAPHS)
def test_standard_mdl(sbp, orc, gs, name):
    g = gs[name]
    for B in (1, 7, 90):
        p = _partition(g, B, B)
        S, d = sbp.mdl(g, p, B, exact=1)
        S_o, d_o = orc.mdl_mode(g, p, B, exact=1)
        assert close(S, S_o) and close(d, d_o)


@pytest.mark.parametrize("name", GRAPHS)
@pytest.mark.parametrize("B", [6, 60])
def test_exact_merge_dS(sbp, orc, gs, name, B):
    g = gs[name]
    p = _partition(g, B, B + 5)
    props = orc.merge_proposals(g, p, B, 11, 0)
    dS, best, bds = sbp.delta_mdl_merge_mode(g, p, B, props, exact=1)
    dS_o, best_o, bds_o = orc.merge_delta_exact(g, p, B, props)
    assert close(dS, dS_o).all()
    assert close(bds, bds_o).all()
    # the best proposal agrees wherever the minimum is not a near tie
    d = dS_o.reshape(B, 10)
    srt = np.sort(d, axis=1)
    clear = (srt[:, 1] - srt[:, 0]) > 1e-6 * np.maximum(np.abs(srt[:, 0]), 1.0)
    assert np.array_equal(best[clear], best_o[clear])


MODES = [(1, 0, 3.0), (1, 1, 3.0), (1, 1, 0.5), (0, 1, 1.0)]


@pytest.mark.parametrize("exact,mh,beta", MODES, ids=[f"x{m[0]}mh{m[1]}b{m[2]}" for m in MODES])
@pytest.mark.parametrize("name", GRAPHS)
def test_nodal_batch_mode_identical(sbp, orc, gs, name, exact, mh, beta):
    g = gs[name]
    B = 30
    p = _partition(g, B, 1)
    BS = g.N // 4
    moved_up = 0
    for b in range(4):
        pa, da, xa, ta = sbp.nodal_batch_mode(g, p, B, 21, 100 + b, b * BS, (b + 1) * BS,
                                              exact=exact, mh=mh, beta=beta)
        pb, db, xb, tb = orc.nodal_batch_mode(g, p, B, 21, 100 + b, b * BS, (b + 1) * BS,
                                              exact=exact, mh=mh, beta=beta)
        assert np.array_equal(xa, xb), "proposals differ"
        assert np.array_equal(pa, pb), "accepted moves differ"
        with np.errstate(invalid="ignore"):
            assert close(da, db).all()
        assert abs(ta - tb) <= REL * max(abs(tb), 1.0)
        moved_up += int((da > 0).sum())
    if not mh:
        assert moved_up == 0
    elif beta < 1.0:
        assert moved_up > 0  # uphill moves accepted


@pytest.mark.parametrize("variant,seed", [("LL", 0), ("HH", 1)])
@pytest.mark.parametrize("exact,mh", [(1, 0), (1, 1)])
def test_partition_exact_mode_matches_oracle(sbp, orc, variant, seed, exact, mh):
    # same draws on both sides; FP64 rounding of exactly tied merges may
    # send the runs down different paths, so the bar is the MDL within 1%
    g = graphs.dcsbm(variant, 1000, 11, seed)
    rep = sbp.partition(g, seed=seed, exact=exact, mh=mh)
    lab_o, rep_o, st = orc.partition(g, seed=seed, exact=exact, mh=mh)
    assert st == 0 and rep["status"] == 0
    # both report the standard description length of their final labels
    assert close(rep["S"], sbp.mdl(g, g.partitions, rep["B"], exact=1)[0])
    assert abs(rep["S"] - rep_o["S"]) <= 0.01 * abs(rep_o["S"])


@pytest.mark.parametrize("exact,mh", [(1, 0), (1, 1), (0, 1)])
def test_partition_exact_mode_same_bits_in_both_forms(sbp, exact, mh):
    g = graphs.dcsbm("HH", 3000, 20, 4)
    out = []
    for dmax in (0, 1024, g.N):
        rep = sbp.partition(g, seed=5, dense_max=dmax, exact=exact, mh=mh)
        out.append((g.partitions.copy(), rep))
    for lab, rep in out[1:]:
        assert np.array_equal(lab, out[0][0])
        assert rep["S"] == out[0][1]["S"] and rep["nodal_itrs"] == out[0][1]["nodal_itrs"]


def test_batch_exact_mode_equals_solo(sbp):
    gl = [graphs.dcsbm(v, 1500, 12, i) for i, v in enumerate(("LL", "HH", "LH"))]
    labs, reps, _ = sbp.partition_batch(gl, seeds=[3, 4, 5], exact=1, mh=1)
    for g, lab, rep, seed in zip(gl, labs, reps, (3, 4, 5)):
        r = sbp.partition(g, seed=seed, exact=1, mh=1)
        assert np.array_equal(lab, g.partitions) and rep["S"] == r["S"]
