"""Command-line partitioner, the counterpart of GSAP's `run <cat> <size>`
(GSAP.cu:7-34): loads or generates a graph, partitions it on the GPU and
prints the run report and the quality against the planted labels as JSON.

    python -m gsap_b200.run --synthetic HH --N 20000 --B 32 [--seed 0]
    python -m gsap_b200.run --tsv graph.tsv [--truth graph_truePartition.tsv]
    python -m gsap_b200.run --dataset /path/to/Dataset/static --cat LL --size 5k
    python -m gsap_b200.run --synthetic HH --N 20000 --B 32 --exact --mh [--beta 3]
"""
import argparse
import json
import sys
import time

from gsap_b200 import sbp


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--synthetic", choices=sorted(sbp.VARIANTS))
    ap.add_argument("--N", type=int, default=20000)
    ap.add_argument("--B", type=int, default=32)
    ap.add_argument("--graph-seed", type=int, default=0)
    ap.add_argument("--tsv")
    ap.add_argument("--truth")
    ap.add_argument("--dataset")
    ap.add_argument("--cat")
    ap.add_argument("--size")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--verbose", "-v", action="count", default=0,
                    help="-v: one line per outer step; -vv: also one line per engine tick; -vvv: also the event-timed segments of every nodal batch")
    ap.add_argument("--dense-max", type=int, default=None,
                    help="largest B kept in the dense blockmodel form")
    ap.add_argument("--exact", action="store_true",
                    help="score moves and merges by the exact change of the MDL")
    ap.add_argument("--mh", action="store_true",
                    help="accept nodal moves by Metropolis-Hastings")
    ap.add_argument("--beta", type=float, default=3.0,
                    help="inverse temperature of the Metropolis-Hastings test, per nat")
    ap.add_argument("--no-phase-timing", action="store_true",
                    help="leave out the per-batch CUDA events that time each phase")
    ap.add_argument("--no-graphs", action="store_true",
                    help="launch the queued sweeps directly instead of as CUDA graphs")
    a = ap.parse_args(argv)
    if a.synthetic:
        g = sbp.dcsbm_variant(a.synthetic, a.N, a.B, seed=a.graph_seed)
    elif a.tsv:
        g = sbp.load_tsv(a.tsv, a.truth)
    elif a.dataset:
        g = sbp.read_file(a.cat, a.size, a.dataset)
    else:
        ap.error("give --synthetic, --tsv or --dataset")
    for i in range(a.repeat):
        t0 = time.perf_counter()
        kw = {} if a.dense_max is None else {"dense_max": a.dense_max}
        kw.update(exact=int(a.exact), mh=int(a.mh), beta=a.beta, use_graphs=int(not a.no_graphs),
                  phase_timing=int(not a.no_phase_timing))
        rep = sbp.partition(g, seed=a.seed + i, device=a.device, verbose=int(a.verbose), **kw)
        rep["wall_ms"] = (time.perf_counter() - t0) * 1000.0
        rep["N"], rep["E"] = g.N, g.E
        # the final labels under both objectives: GSAP's MDL formula and the
        # standard description length (exact mode's)
        rep["S_gsap_formula"] = sbp.mdl(g, g.partitions, rep["B"])[0]
        rep["S_standard"] = sbp.mdl(g, g.partitions, rep["B"], exact=1)[0]
        if g.true_partitions is not None and g.true_partitions.min() >= 0:
            r, p, n = sbp.evaluate(g.true_partitions, g.partitions)
            rep.update(recall=r, precision=p, nmi=n)
        print(json.dumps(rep), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
