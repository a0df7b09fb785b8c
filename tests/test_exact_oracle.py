"""The oracle's exact-MDL mode against brute force.

Exact mode scores a move by the true change of the description length:
with B fixed, S(after) - S(before) of the full MDL (the model term does not
move), so every dS it gives must equal the difference of two full MDL
evaluations of the partitions before and after the move.  The Hastings
ratio is checked against a direct evaluation of GSAP's proposal
probability p(s | t) = (M_ts + M_st + 1) / (d_t + B), averaged over v's
edges (a self loop counts once per direction), before and after the move.
"""
import numpy as np
import pytest

import graphs


def _self_loop_graph(sbp, N=300, seed=5):
    rng = np.random.default_rng(seed)
    E = N * 6
    src = rng.integers(0, N, E).astype(np.int32)
    dst = rng.integers(0, N, E).astype(np.int32)
    loops = rng.choice(N, N // 5, replace=False).astype(np.int32)
    src = np.concatenate([src, loops])
    dst = np.concatenate([dst, loops])
    w = rng.integers(1, 4, src.size).astype(np.uint32)
    order = np.argsort(src, kind="stable")
    return sbp.Graph.from_edges(N, src[order], dst[order], w[order])


def _cases(sbp):
    return [("LL", graphs.dcsbm("LL", 600, 9, seed=1)),
            ("weighted", graphs.weighted_graph(400, seed=3)),
            ("self_loops", _self_loop_graph(sbp))]


def _block_matrix(g, part, B):
    src, dst, w = g.edges()
    M = np.zeros((B, B))
    np.add.at(M, (part[src], part[dst]), w.astype(np.float64))
    return M


def _hastings_direct(g, part, B, v, s):
    src, dst, w = g.edges()
    r = part[v]
    if r == s:
        return 0.0

    def p_of(pt, target):
        M = _block_matrix(g, pt, B)
        dt = M.sum(axis=0) + M.sum(axis=1)
        tot, num = 0.0, 0.0
        for sel, other in ((src == v, dst), (dst == v, src)):
            for u, ww in zip(other[sel], w[sel]):
                t = pt[u]
                num += ww * (M[t, target] + M[target, t] + 1.0) / (dt[t] + B)
                tot += ww
        return num / tot

    if (src == v).sum() + (dst == v).sum() == 0:
        return 0.0
    after = part.copy()
    after[v] = s
    return np.log(p_of(after, r)) - np.log(p_of(part, s))


@pytest.mark.parametrize("name", ["LL", "weighted", "self_loops"])
def test_exact_nodal_dS_is_the_mdl_difference(sbp, orc, name):
    g = dict(_cases(sbp))[name]
    rng = np.random.default_rng(7)
    for B in (3, 17, 60):
        part = rng.integers(0, B, g.N).astype(np.int32)
        part[:B] = np.arange(B, dtype=np.int32)
        verts = rng.choice(g.N, 40, replace=False).astype(np.int32)
        props = rng.integers(0, B, verts.size).astype(np.int32)
        dS, _ = orc.nodal_delta_exact(g, part, B, verts, props)
        S0, _ = orc.mdl(g, part, B)
        for i, v in enumerate(verts):
            after = part.copy()
            after[v] = props[i]
            S1, _ = orc.mdl(g, after, B)
            assert abs(dS[i] - (S1 - S0)) <= 1e-9 * max(1.0, abs(S0)), (B, v)


@pytest.mark.parametrize("name", ["LL", "weighted", "self_loops"])
def test_exact_merge_dS_is_the_mdl_difference(sbp, orc, name):
    g = dict(_cases(sbp))[name]
    rng = np.random.default_rng(8)
    for B in (4, 25):
        part = rng.integers(0, B, g.N).astype(np.int32)
        part[:B] = np.arange(B, dtype=np.int32)
        props = orc.merge_proposals(g, part, B, 11, 0)
        dS, best, bds = orc.merge_delta_exact(g, part, B, props)
        S0, _ = orc.mdl(g, part, B)
        for t in range(0, B * 10, 3):
            r, s = t // 10, props[t]
            after = np.where(part == r, s, part).astype(np.int32)
            S1, _ = orc.mdl(g, after, B)
            want = 0.0 if r == s else S1 - S0
            assert abs(dS[t] - want) <= 1e-9 * max(1.0, abs(S0)), (B, r, s)
        # best is the minimum over each block's proposals
        assert np.allclose(bds, dS.reshape(B, 10).min(axis=1))


@pytest.mark.parametrize("name", ["weighted", "self_loops"])
def test_hastings_ratio_matches_direct_evaluation(sbp, orc, name):
    g = dict(_cases(sbp))[name]
    rng = np.random.default_rng(9)
    B = 12
    part = rng.integers(0, B, g.N).astype(np.int32)
    part[:B] = np.arange(B, dtype=np.int32)
    verts = rng.choice(g.N, 25, replace=False).astype(np.int32)
    props = rng.integers(0, B, verts.size).astype(np.int32)
    _, lh = orc.nodal_delta_exact(g, part, B, verts, props)
    for i, v in enumerate(verts):
        assert abs(lh[i] - _hastings_direct(g, part, B, v, props[i])) <= 1e-12, (v, props[i])


def test_mh_batch_accepts_uphill_moves_and_quirk_mode_does_not(sbp, orc):
    g = graphs.dcsbm("LL", 2000, 11, seed=2)
    rng = np.random.default_rng(4)
    B = 40
    part = rng.integers(0, B, g.N).astype(np.int32)
    part[:B] = np.arange(B, dtype=np.int32)
    _, dS_q, _, _ = orc.nodal_batch_mode(g, part, B, 3, 0, 0, g.N, exact=1, mh=0)
    _, dS_m, _, _ = orc.nodal_batch_mode(g, part, B, 3, 0, 0, g.N, exact=1, mh=1, beta=1.0)
    assert (dS_q <= 0).all()
    assert (dS_m > 0).any()
    # MH mode records the accepted moves' exact dS, greedy mode only downhill
    p_m, _, props, _ = orc.nodal_batch_mode(g, part, B, 3, 0, 0, g.N, exact=1, mh=1, beta=1.0)
    moved = p_m != part
    assert np.array_equal(p_m[moved], props[moved])


def test_standard_mdl_formula(sbp, orc):
    # exact mode's objective: (E h(B^2/E) + N ln B) / ln 2 - data_S, in bits
    g = graphs.dcsbm("LH", 1500, 9, seed=3)
    rng = np.random.default_rng(1)
    for B in (1, 9, 40):
        p = rng.integers(0, B, g.N).astype(np.int32)
        p[:B] = np.arange(B, dtype=np.int32)
        M = _block_matrix(g, p, B)
        dout, din = M.sum(axis=1), M.sum(axis=0)
        nz = M > 0
        data = (M[nz] * np.log2(M[nz])).sum() - (dout[dout > 0] * np.log2(dout[dout > 0])).sum() \
            - (din[din > 0] * np.log2(din[din > 0])).sum()
        x = B * B / g.E
        model = (g.E * ((1 + x) * np.log(1 + x) - x * np.log(x)) + g.N * np.log(B)) / np.log(2)
        S, d = orc.mdl_mode(g, p, B, exact=1)
        assert abs(d - data) <= 1e-9 * abs(data)
        assert abs(S - (model - data)) <= 1e-9 * abs(S)
        # GSAP's formula (exact = 0) keeps its own model term and the same data_S
        S6, d6 = orc.mdl_mode(g, p, B, exact=0)
        assert d6 == d and (S6, d6) == orc.mdl(g, p, B)
