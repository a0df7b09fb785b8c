"""Seeded test graphs (DCSBM variants plus hand-built shapes that reach
every path of the blockmodel builder and the dS kernels)."""
import numpy as np

from gsap_b200 import sbp


def dcsbm(variant="LL", N=1000, B=11, seed=0):
    return sbp.dcsbm_variant(variant, N, B, seed=seed)


def hub_graph(N=20000, hub_in=9000, seed=1):
    """A DCSBM graph plus one vertex with `hub_in` extra in-edges and a
    second with 1000, so that at B = N their in-rows are longer than a
    warp's sort buffer and longer than a CTA's."""
    g = sbp.dcsbm(N, 32, 1.0, 0.5, seed=seed)
    src, dst, w = g.edges()
    rng = np.random.default_rng(seed)
    extra = []
    for hub, k in ((0, hub_in), (1, 1000)):
        s = rng.choice(np.arange(2, N), size=k, replace=False).astype(np.int32)
        have = set(src[dst == hub].tolist())
        s = np.array([x for x in s if x not in have], np.int32)
        extra.append((s, np.full(s.size, hub, np.int32)))
    src = np.concatenate([src] + [e[0] for e in extra])
    dst = np.concatenate([dst] + [e[1] for e in extra])
    return sbp.Graph.from_edges(N, src, dst, None, g.true_partitions)


def weighted_graph(N=600, seed=2):
    """Non-unit weights and repeated (u, v) pairs."""
    rng = np.random.default_rng(seed)
    E = N * 8
    src = rng.integers(0, N, E).astype(np.int32)
    dst = rng.integers(0, N, E).astype(np.int32)
    keep = src != dst
    src, dst = src[keep], dst[keep]
    w = rng.integers(1, 5, src.size).astype(np.uint32)
    order = np.argsort(src, kind="stable")
    return sbp.Graph.from_edges(N, src[order], dst[order], w[order])


def partitions(g, seed=0):
    """(name, labels, B) cases: every vertex alone, the planted labels, and
    random labelings at several B."""
    rng = np.random.default_rng(seed)
    out = [("identity", np.arange(g.N, dtype=np.int32), g.N)]
    if g.true_partitions is not None and g.true_partitions.min() >= 0:
        t = g.true_partitions.astype(np.int32)
        out.append(("planted", t, int(t.max()) + 1))
    for B in (7, 40, max(2, g.N // 10)):
        p = rng.integers(0, B, g.N).astype(np.int32)
        p[:B] = np.arange(B, dtype=np.int32)  # no empty block
        out.append((f"random{B}", p, B))
    return out
