"""Graph ingest on the device: sbp_dcsbm_generate_device and
sbp_graph_from_device_edges against the oracle.

The generator must give the oracle's DCSBM graph (orc_dcsbm, pinned to the
host generator by test_oracle_generator.py) edge for edge, and the device CSR
build must give the CSR pair the oracle builds with load.hpp's ordering
(GSAP/load.hpp:86-117: rows in input edge order) on the same edges: bit for
bit in every array.  Edge lists cover unsorted input, repeated edges, self
loops, weights, a hub row of 133k entries, E = 0 and N = 1; bad endpoints
and zero weights come back as SBP_ERR_INVALID.  A graph built on the device
partitions to the same labels as the same graph uploaded from the host."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS = ("out_ptr", "out_idx", "out_w", "in_ptr", "in_idx", "in_w", "deg_out", "deg_in")


def _same_csr(a, b):
    for k in KEYS:
        x, y = np.asarray(getattr(a, k)), np.asarray(getattr(b, k))
        assert x.shape == y.shape, (k, x.shape, y.shape)
        assert np.array_equal(x.astype(np.int64), y.astype(np.int64)), k


GEN_CASES = [
    # N, B, alpha, p_in, deg_min, deg_max, exponent, seed
    (200000, 71, 1.0, 0.5, 5, 50, 2.5, 0),    # the 200k HH benchmark graph
    (20000, 32, 20.0, 0.8, 5, 50, 2.5, 3),    # LL
    (20000, 32, 1.0, 0.8, 5, 50, 2.5, 4),     # LH
    (20000, 32, 20.0, 0.5, 5, 50, 2.5, 5),    # HL
    (5000, 1, 1.0, 0.5, 1, 20, 2.0, 1),       # one block
    (300, 300, 0.5, 0.0, 2, 9, 1.5, 2),       # every vertex its own block, no in-block edges
    (64, 4, 3.0, 1.0, 1, 63, 0.5, 9),         # deg_max = N - 1: many draws fail
]


@pytest.mark.parametrize("case", GEN_CASES, ids=lambda c: f"N{c[0]}B{c[1]}s{c[7]}")
def test_device_generator_matches_oracle(sbp, orc, case):
    N, B, alpha, p_in, dmin, dmax, ex, seed = case
    ref = orc.dcsbm(N, B, alpha, p_in, seed=seed, deg_min=dmin, deg_max=dmax, exponent=ex)
    dg = sbp.dcsbm_device(N, B, alpha, p_in, seed=seed, deg_min=dmin, deg_max=dmax,
                          exponent=ex, device=0)
    try:
        assert (dg.N, dg.E) == (ref.N, ref.E)
        assert np.array_equal(dg.true_partitions, ref.true_partitions)
        _same_csr(dg.download(), ref)
    finally:
        dg.close()


def _edges_on_device(src, dst, w):
    import torch
    ts = torch.from_numpy(np.ascontiguousarray(src, np.int32)).cuda()
    td = torch.from_numpy(np.ascontiguousarray(dst, np.int32)).cuda()
    tw = None if w is None else torch.from_numpy(np.ascontiguousarray(w, np.uint32).view(np.int32)).cuda()
    return ts, td, tw


def _edge_cases():
    rng = np.random.default_rng(11)
    out = []
    N = 3000
    E = 40000
    out.append(("random", N, rng.integers(0, N, E), rng.integers(0, N, E), None))
    src = rng.integers(0, N, E)
    dst = rng.integers(0, N, E)
    dst[:500] = src[:500]                     # self loops
    src[500:1500] = 7                          # one long out-row
    dst[1000:1200] = 9                         # repeated edge (7, 9)
    w = rng.integers(1, 1000, E)
    out.append(("weighted_loops_repeats", N, src, dst, w))
    N = 200000
    E = 400000
    src = rng.integers(0, N, E)
    dst = rng.integers(0, N, E)
    dst[::3] = 12345                           # a hub of ~133k in-entries
    out.append(("hub", N, src, dst, None))
    out.append(("empty", 50, np.zeros(0, np.int64), np.zeros(0, np.int64), None))
    out.append(("one_vertex", 1, np.zeros(5, np.int64), np.zeros(5, np.int64),
                np.array([1, 2, 3, 4, 5])))
    return out


@pytest.mark.parametrize("case", _edge_cases(), ids=lambda c: c[0])
def test_device_csr_build_matches_oracle(sbp, orc, case):
    name, N, src, dst, w = case
    ref = orc.Graph(N, src, dst, w)
    ts, td, tw = _edges_on_device(src, dst, w)
    E = int(len(src))
    dg = sbp.DeviceGraph.from_edges(N, ts.data_ptr() if E else 0, td.data_ptr() if E else 0, E,
                                    None if tw is None else tw.data_ptr(), device=0)
    try:
        assert (dg.N, dg.E) == (N, E)
        _same_csr(dg.download(), ref)
        # and the host builder (sbp_csr_from_edges) agrees
        _same_csr(dg.download(), sbp.Graph.from_edges(N, src, dst, w))
    finally:
        dg.close()


@pytest.mark.parametrize("bad", ["src_high", "dst_negative", "zero_weight"])
def test_device_csr_build_rejects_bad_edges(sbp, bad):
    rng = np.random.default_rng(5)
    N, E = 100, 1000
    src = rng.integers(0, N, E)
    dst = rng.integers(0, N, E)
    w = rng.integers(1, 5, E)
    if bad == "src_high":
        src[17] = N
    elif bad == "dst_negative":
        dst[400] = -3
    else:
        w[999] = 0
    ts, td, tw = _edges_on_device(src, dst, w)
    with pytest.raises(sbp.SbpError) as ei:
        sbp.DeviceGraph.from_edges(N, ts.data_ptr(), td.data_ptr(), E, tw.data_ptr(), device=0)
    assert ei.value.status == 1


def test_device_graph_partitions_like_host_graph(sbp):
    g = sbp.dcsbm_variant("HH", 20000, 32, seed=1)
    dg = sbp.dcsbm_variant_device("HH", 20000, 32, seed=1, device=0)
    try:
        lab_d, rep_d = dg.partition(seed=3)
        lab_h, rep_h = sbp.ResidentGraph(g, device=0).partition(seed=3)
        assert np.array_equal(lab_d, lab_h)
        assert rep_d["S"] == rep_h["S"] and rep_d["B"] == rep_h["B"]
        # options that grow the job's arena rebuild the CSR from the device edges
        lab_g, rep_g = dg.partition(seed=3, num_proposals=12)
        rep_gh = sbp.partition(g, seed=3, num_proposals=12)
        assert np.array_equal(lab_g, g.partitions) and rep_g["S"] == rep_gh["S"]
    finally:
        dg.close()
