"""GPU path vs the CPU oracle on the benchmark graphs themselves: the four
20k-vertex variants (LL, LH, HL, HH; 32 planted blocks) and the 200k-vertex
HH graph (71 planted blocks), seed 0.

For each graph, at three labelings the run passes through (every vertex
alone, B = N; after GSAP's first merge step, B = 0.65 N; the planted
blocks):
  * the blockmodel is bit-exact;
  * one nodal batch (the first quarter of the vertices) draws the same
    proposals, accepts the same moves and records dS within 1e-9, relative
    to the value or, for moves of the giant block GSAP's first merge step
    makes, to the magnitude of the row sums the oracle's value is the
    difference of (1e-12 of it: the FP64 rounding of those sums; the GPU's
    formulation does not subtract them);
  * one merge step gives the same best dS per block within 1e-9 and, where
    the two rankings agree, the same labels.
The first merge step reproduces GSAP's merge grid (the proposal slots past
the nnz of the out CSR read fresh zeros), as the partitioner's default does.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL = 1e-9
CONFIGS = [("LL", 20000, 32), ("LH", 20000, 32), ("HL", 20000, 32), ("HH", 20000, 32),
           ("HH", 200000, 71)]
IDS = [f"{v}{N // 1000}k" for v, N, _ in CONFIGS]
KEYS = ("optr", "ocol", "ocnt", "iptr", "icol", "icnt", "d_out", "d_in")


def close(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    with np.errstate(invalid="ignore"):
        return (a == b) | (np.abs(a - b) <= REL * np.maximum(np.abs(b), 1.0))


_CACHE = {}


def setup(sbp, orc, cfg):
    """The graph and its three labelings (identity, after the first merge
    step, planted), computed once per config."""
    if cfg not in _CACHE:
        v, N, B = cfg
        g = sbp.dcsbm_variant(v, N, B, seed=0)
        ident = np.arange(g.N, dtype=np.int32)
        k = int(np.float32(g.N) * np.float32(0.35))
        merged, nb, best, bds = orc.merge_step(g, ident, g.N, k, seed=0, seq=0, ref_grid=1)
        planted = g.true_partitions.astype(np.int32)
        _CACHE[cfg] = (g, [("identity", ident, g.N), ("first-merge", merged, nb),
                           ("planted", planted, int(planted.max()) + 1)],
                       (best, bds, merged, nb, k))
    return _CACHE[cfg]


@pytest.mark.parametrize("cfg", CONFIGS, ids=IDS)
def test_blockmodel_bit_exact_at_configs(sbp, orc, cfg):
    g, labs, _ = setup(sbp, orc, cfg)
    for name, p, B in labs:
        a = sbp.build_blockmodel(g, p, B)
        b = orc.build_blockmodel(g, p, B)
        for key in KEYS:
            assert np.array_equal(a[key], b[key]), (name, key)


@pytest.mark.parametrize("cfg", CONFIGS, ids=IDS)
def test_nodal_batch_at_configs(sbp, orc, cfg):
    g, labs, _ = setup(sbp, orc, cfg)
    BS = g.N // 4
    for name, p, B in labs[1:]:
        pa, da, xa, ta = sbp.nodal_batch(g, p, B, 21, 100, 0, BS)
        pb, db, xb, tb = orc.nodal_batch(g, p, B, 21, 100, 0, BS)
        assert np.array_equal(xa, xb), (name, "proposals differ")
        _, mag = orc.nodal_delta_scale(g, p, B, np.arange(BS, dtype=np.int32), xb)
        ok = close(da, db) | (np.abs(da - db) <= 1e-12 * mag)
        bad = np.flatnonzero(~ok)
        assert ok.all(), (name, bad[:5], da[bad[:5]], db[bad[:5]], p[bad[:5]], xb[bad[:5]])
        # a move whose dS is zero in exact arithmetic may land on either side
        # of zero after rounding; every other decision must agree
        diff = np.flatnonzero(pa != pb)
        if diff.size:
            raw, _ = orc.nodal_delta(g, p, B, diff.astype(np.int32), xb[diff])
            assert (np.abs(raw) <= REL).all(), (name, diff[:5], raw[:5])
        assert abs(ta - tb) <= REL * max(abs(tb), 1.0), name
        if name == "first-merge":
            assert (db < 0).sum() > 0  # the batch does move vertices


@pytest.mark.parametrize("cfg", CONFIGS, ids=IDS)
def test_first_merge_step_at_configs(sbp, orc, cfg):
    # GSAP's first merge step (B = N): the blocks past its merge grid
    # propose block 0 with dS 0 and merge into it first
    g, labs, (best_o, bds_o, merged_o, nb_o, k) = setup(sbp, orc, cfg)
    ident = labs[0][1]
    pa, nba, ba, bda = sbp.merge_step(g, ident, g.N, k, seed=0, seq=0, ref_grid=1)
    assert close(bda, bds_o).all()
    T = (g.E + 255) // 256 * 256  # nnz = E at B = N (no repeated edges)
    tail = np.arange(g.N) >= -(-T // 10)
    assert tail.any() and (ba[tail] == 0).all() and (bda[tail] == 0).all()
    ties = ba != best_o
    for r in np.flatnonzero(ties):
        assert close(bda[r], bds_o[r]), r
    if not ties.any():
        assert nba == nb_o and np.array_equal(pa, merged_o)
    # without the grid every block gets its own proposals
    pc, nbc, bc, bdc = sbp.merge_step(g, ident, g.N, k, seed=0, seq=0, ref_grid=0)
    assert not (bc[tail] == 0).all()


@pytest.mark.parametrize("cfg", CONFIGS, ids=IDS)
def test_merge_step_at_planted(sbp, orc, cfg):
    g, labs, _ = setup(sbp, orc, cfg)
    _, p, B = labs[2]
    k = max(1, int(B * 0.35))
    pa, nba, ba, bda = sbp.merge_step(g, p, B, k, seed=4, seq=1)
    pb, nbb, bb, bdb = orc.merge_step(g, p, B, k, seed=4, seq=1)
    assert close(bda, bdb).all()
    pc, nbc = orc.apply_merges(p, B, k, ba, bda)
    assert nba == nbc and np.array_equal(pa, pc)
    if np.array_equal(ba, bb):
        assert nba == nbb and np.array_equal(pa, pb)
