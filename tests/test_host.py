"""Host-side pieces of the C ABI (no GPU): the library loads and exports
every symbol include/sbp.h declares, the loader reads GraphChallenge TSVs
exactly as GSAP/load.hpp does, the CSR builder, the DCSBM generator, and
input validation that runs before any device call."""
import hashlib
import json
import os
import re

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _dataset_dir():
    """The GraphChallenge graphs bundled with the reference tree: under $REF,
    else under the tree oracle/build_ref.sh built the checkers from (its
    oracle/_ref/ref_root).  Empty when neither is on this machine."""
    ref = os.environ.get("REF", "")
    marker = os.path.join(ROOT, "oracle", "_ref", "ref_root")
    if not ref and os.path.exists(marker):
        ref = open(marker).read().strip()
    return os.path.join(ref, "Dataset", "static") if ref else ""


DATA = _dataset_dir()


def test_exports_every_declared_symbol(sbp):
    hdr = open(os.path.join(ROOT, "include", "sbp.h")).read()
    declared = set(re.findall(r"^\w[\w\s\*]*?\b(sbp_\w+)\s*\(", hdr, re.M))
    assert declared, "no declarations parsed"
    import ctypes
    lib = ctypes.CDLL(sbp.LIB_PATH)
    for name in sorted(declared):
        assert hasattr(lib, name), name
    assert declared <= set(sbp.EXPORTED) | declared


def test_default_options_are_gsaps(sbp):
    o = sbp.default_options()
    # partition.hpp:855-861
    assert o.num_proposals == 10 and abs(o.reduction_rate - 0.35) < 1e-7
    assert o.max_nodal_itr == 100 and o.num_batches == 4 and o.window == 3
    assert abs(o.threshold1 - 5e-4) < 1e-10 and abs(o.threshold2 - 1e-4) < 1e-10
    # GSAP's scoring: its dS terms, accept iff dS < 0
    assert o.exact == 0 and o.mh == 0 and o.beta == 3.0


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.skipif(not os.path.isdir(DATA), reason="GraphChallenge fixtures not present")
@pytest.mark.parametrize("cat", ["LL", "LH", "HL", "HH"])
@pytest.mark.parametrize("size", ["1k", "5k"])
def test_loader_matches_reference(sbp, cat, size):
    gold = json.load(open(os.path.join(HERE, "golden", "loader.json")))[f"{cat}-{size}"]
    g = sbp.read_file(cat, size, DATA)
    assert (g.N, g.E) == (gold["N"], gold["E"])
    # the reference keeps N row pointers (no end sentinel)
    assert _sha(g.out_ptr[:-1]) == gold["out_ptr"]
    assert _sha(g.in_ptr[:-1]) == gold["in_ptr"]
    for k in ("out_idx", "out_w", "in_idx", "in_w", "deg_out", "deg_in"):
        assert _sha(getattr(g, k)) == gold[k], k
    assert _sha(g.true_partitions) == gold["truth"]


def test_loader_first_field_with_space(sbp, tmp_path):
    # load.hpp:50-65: "1 408\t1" parses as the self-loop (1, 1, 1)
    p = tmp_path / "g.tsv"
    p.write_text("1 408\t1\n1\t2\t1\n2\t1\t3\n")
    g = sbp.load_tsv(str(p))
    src, dst, w = g.edges()
    assert g.N == 2 and g.E == 3
    assert list(zip(src, dst, w)) == [(0, 0, 1), (0, 1, 1), (1, 0, 3)]


def test_csr_from_edges_keeps_edge_order(sbp):
    src = np.array([2, 0, 2, 1, 0], np.int32)
    dst = np.array([0, 2, 1, 0, 1], np.int32)
    w = np.array([1, 2, 3, 4, 5], np.uint32)
    g = sbp.Graph.from_edges(3, src, dst, w)
    assert list(g.out_ptr) == [0, 2, 3, 5]
    assert list(g.out_idx) == [2, 1, 0, 0, 1] and list(g.out_w) == [2, 5, 4, 1, 3]
    assert list(g.in_ptr) == [0, 2, 4, 5]
    assert list(g.in_idx) == [2, 1, 2, 0, 0]
    assert list(g.deg_out) == [7, 4, 4] and list(g.deg_in) == [5, 8, 2]


def test_dcsbm_is_deterministic_and_has_its_shape(sbp):
    a = sbp.dcsbm_variant("HH", 20000, 32, seed=4)
    b = sbp.dcsbm_variant("HH", 20000, 32, seed=4)
    c = sbp.dcsbm_variant("HH", 20000, 32, seed=5)
    assert np.array_equal(a.out_idx, b.out_idx) and np.array_equal(a.true_partitions,
                                                                   b.true_partitions)
    assert not np.array_equal(a.true_partitions, c.true_partitions)
    t = a.true_partitions
    assert t.min() == 0 and t.max() == 31 and np.bincount(t).min() >= 1
    src, dst, _ = a.edges()
    assert not np.any(src == dst), "self-loop"
    key = src.astype(np.int64) * a.N + dst
    assert np.unique(key).size == key.size, "repeated edge"
    deg = np.diff(a.out_ptr)
    assert deg.min() >= 5 and deg.max() <= 50
    assert 9.0 < a.E / a.N < 10.5  # truncated power law 2.5 on [5, 50]: mean 9.78
    frac_in = np.mean(t[src] == t[dst])
    assert abs(frac_in - 0.5) < 0.02  # p_in of HH
    ll = sbp.dcsbm_variant("LL", 20000, 32, seed=4)
    s2, d2, _ = ll.edges()
    assert abs(np.mean(ll.true_partitions[s2] == ll.true_partitions[d2]) - 0.8) < 0.02
    # alpha = 20 gives near-equal block sizes, alpha = 1 spread ones
    assert np.bincount(ll.true_partitions).std() < np.bincount(t).std()


def test_evaluate_rejects_bad_labels(sbp):
    with pytest.raises(sbp.SbpError):
        sbp.evaluate(np.zeros(4, np.int32), np.array([0, -1, 0, 0], np.int32))


def test_partition_validates_before_device_use(sbp):
    g = sbp.dcsbm_variant("LL", 1000, 11, seed=0)
    bad = sbp.Graph(**{**g.__dict__, "deg_out": g.deg_out + 1})
    with pytest.raises(sbp.SbpError, match="invalid argument"):
        sbp.partition(bad)
    with pytest.raises(sbp.SbpError, match="invalid argument"):
        sbp.partition(g, num_proposals=0)
    with pytest.raises(sbp.SbpError, match="invalid argument"):
        sbp.build_blockmodel(g, np.full(g.N, 11, np.int32), 11)
    with pytest.raises(sbp.SbpError, match="invalid argument"):
        sbp.delta_mdl_nodal(g, g.true_partitions, 11, [0], [11])
    # scoring modes
    with pytest.raises(sbp.SbpError, match="invalid argument"):
        sbp.partition(g, exact=2)
    with pytest.raises(sbp.SbpError, match="invalid argument"):
        sbp.partition(g, mh=1, beta=-1.0)
    with pytest.raises(sbp.SbpError, match="invalid argument"):
        sbp.nodal_batch_mode(g, g.true_partitions, 11, 0, 0, 0, 10, exact=3)
    with pytest.raises(sbp.SbpError, match="invalid argument"):
        sbp.delta_mdl_nodal_mode(g, g.true_partitions, 11, [0], [1], exact=-1)
    with pytest.raises(sbp.SbpError, match="invalid argument"):
        sbp.delta_mdl_merge_mode(g, g.true_partitions, 11, np.zeros(110, np.int32), exact=2)


def test_validation_reports_the_first_error_in_order(sbp):
    # large enough that the entries are checked by several host threads; the
    # error reported is still the first in (direction, vertex) order
    g = sbp.dcsbm_variant("HH", 120000, 20, seed=1)
    assert g.E > 4 * 262144

    def bad(**arrays):
        fields = {**g.__dict__}
        for k, v in arrays.items():
            fields[k] = v
        with pytest.raises(sbp.SbpError) as e:
            sbp.partition(sbp.Graph(**fields))
        return str(e.value)

    late_out = g.out_idx.copy()
    late_out[-1] = g.N + 5  # direction 0, last vertex
    early_in_w = g.in_w.copy()
    early_in_w[0] = 0  # direction 1, first vertex
    msg = bad(out_idx=late_out, in_w=early_in_w)
    assert "vertex id out of range" in msg
    msg = bad(in_w=early_in_w)
    assert "edge weights must be >= 1" in msg
    deg = g.deg_in.copy()
    deg[-1] += 1
    assert "node degree differs" in bad(deg_in=deg)
    ptr = g.out_ptr.copy()
    ptr[g.N // 2] = ptr[g.N // 2 + 1] + 1
    assert "row pointers decrease" in bad(out_ptr=ptr, in_w=early_in_w)


def test_dense_crossover_grows_with_the_edge_count(sbp):
    # the default dense_max (-1) keeps the dense B x B form while
    # B <= max(4096, sqrt(32 E)), at most N; the job arena holds two B x B
    # uint32 matrices and their row chunk sums at that cap
    def dense_bytes(cap):
        r = lambda b: (b + 255) // 256 * 256
        return 2 * r(cap * cap * 4) + r(2 * cap * ((cap + 31) // 32) * 4)

    def extra(N, E, **kw):
        return sbp.job_bytes(N, E, **kw) - sbp.job_bytes(N, E, dense_max=0)

    assert extra(200000, 2000000) == dense_bytes(8000)  # sqrt(32 * 2e6) = 8000
    assert extra(200000, 2000000, dense_max=4096) == dense_bytes(4096)
    assert extra(20000, 200000) == dense_bytes(4096)    # small graphs keep 4096
    assert extra(3000, 40000) == dense_bytes(3000)      # never above N


@pytest.mark.parametrize("B", [1, 7, 300, 5000, 70000])
def test_apply_merges_matches_oracle(sbp, orc, B):
    # carry_out_best_merges on the host (radix-ranked, threaded for large B)
    # against the oracle's literal loop, with tied, signed-zero and NaN dS
    rng = np.random.default_rng(B)
    for trial in range(4):
        best = rng.integers(0, B, B).astype(np.int32)
        kind = rng.integers(0, 6, B)
        ds = np.ldexp(rng.integers(-10**6, 10**6, B).astype(np.float64), -rng.integers(0, 40, B))
        ds[kind == 0] = 0.0
        ds[kind == 1] = -0.0
        ds[kind == 2] = np.nan
        ds[kind == 3] = rng.integers(0, 4, int((kind == 3).sum()))
        k = int(rng.integers(0, B + 1))
        part = rng.integers(0, B, 4 * B).astype(np.int32)
        m, nb = sbp.apply_merges(B, k, best, ds)
        want, nb_o = orc.apply_merges(part, B, k, best, ds)
        assert nb == nb_o
        assert np.array_equal(m[part], want)
    with pytest.raises(sbp.SbpError, match="invalid argument"):
        sbp.apply_merges(B, 1, np.full(B, B, np.int32), np.zeros(B))
