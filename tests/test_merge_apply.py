"""Merge application on the GPU (mergeapply.cu, the partition loop's path)
against the oracle's literal carry_out_best_merges loop (partition.hpp:26-78):
the same map and block count bit for bit, with tied, signed-zero and NaN dS,
long chains, long cycles and self-proposals."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _check(sbp, orc, B, k, best, ds):
    m, nb = sbp.apply_merges_device(B, k, best, ds)
    ident = np.arange(B, dtype=np.int32)
    want, nb_o = orc.apply_merges(ident, B, k, best, ds)
    assert nb == nb_o
    assert np.array_equal(m, want)


@pytest.mark.parametrize("B", [1, 2, 7, 300, 4096, 4097, 5000, 70000, 200000])
def test_device_merges_match_oracle(sbp, orc, B):
    rng = np.random.default_rng(B + 1)
    for trial in range(3):
        best = rng.integers(0, B, B).astype(np.int32)
        kind = rng.integers(0, 6, B)
        ds = np.ldexp(rng.integers(-10**6, 10**6, B).astype(np.float64),
                      -rng.integers(0, 40, B))
        ds[kind == 0] = 0.0
        ds[kind == 1] = -0.0
        ds[kind == 2] = np.nan
        ds[kind == 3] = rng.integers(0, 4, int((kind == 3).sum()))
        for k in (0, int(B * 0.35), int(rng.integers(0, B + 1)), B):
            _check(sbp, orc, B, k, best, ds)


@pytest.mark.parametrize("B", [1000, 4096, 100000])
def test_device_merges_chains_and_cycles(sbp, orc, B):
    rng = np.random.default_rng(7)
    ds = rng.standard_normal(B)
    ar = np.arange(B, dtype=np.int32)
    shapes = {
        "chain": np.minimum(ar + 1, B - 1).astype(np.int32),      # one path, self at the end
        "cycle": ((ar + 1) % B).astype(np.int32),                 # one cycle of length B
        "self": ar.copy(),                                        # every block proposes itself
        "pairs": (ar ^ 1).clip(0, B - 1).astype(np.int32),        # mutual pairs
        "star": np.zeros(B, np.int32),                            # everything into block 0
    }
    for name, best in shapes.items():
        for k in (1, B // 3, B - 1, B):
            _check(sbp, orc, B, k, best, ds)
        _check(sbp, orc, B, B // 2, best, np.zeros(B))  # all tied: block order


def test_device_merges_from_real_merge_step(sbp, orc):
    # best targets and dS of an actual merge step (identity and planted labels)
    from gsap_b200 import sbp as s
    g = s.dcsbm_variant("HH", 20000, 32, seed=0)
    for p, B in ((np.arange(g.N, dtype=np.int32), g.N),
                 (g.true_partitions.astype(np.int32), 32)):
        props = orc.merge_proposals(g, p, B, seed=3, seq=1)
        _, best, bds = orc.merge_delta(g, p, B, props)
        for k in (int(B * 0.35), B // 2):
            _check(sbp, orc, B, k, best, bds)


def test_device_merges_reject_bad_target(sbp):
    with pytest.raises(sbp.SbpError, match="out of"):
        sbp.apply_merges_device(10, 1, np.full(10, 10, np.int32), np.zeros(10))
