"""The golden-section search over B (GSAP/partition.hpp:80-322), step by step.

Full runs of the GPU and of the oracle part ways after the first merges
(merge dS that tie in exact arithmetic rank differently under different
FP64 summation orders), so their traces are not compared with each other.
Instead each run's trace is checked against the search's own rule: after
every outer step, the bracket (large, med, small) takes the step's (B, S)
and fixes the next B (or ends the search), and the next step of the run
must have exactly that B.  `replay` restates the bookkeeping of
partition.hpp:80-322 as the oracle's run_partition writes it; the CPU test
pins it to the oracle's own trace (orc_partition_trace), the GPU test holds
the engine's trace (its `-v` step lines) to it, including the step at which
the search ends."""
import math
import re

import numpy as np
import pytest

import graphs


def replay(steps, N, rate=0.35):
    """The B that the search picks after each step of `steps` (a list of (B,
    S, ...)), None where it declares the search done.  The first merge takes
    B_to_merge = (float)N * rate blocks away (float32, truncated), as do the
    steps while the bracket has no small end; then
    next_B = med.B + round((large.B - med.B) * 0.618) from the larger side,
    or small.B + round((med.B - small.B) * 0.618), and the search ends when
    large.B - small.B == 2 or nothing is left to merge."""
    inf = math.inf
    large, med, small = (0, inf), (0, inf), (0, inf)
    r32 = np.float32(rate)
    want = []
    for step in steps:
        P = (step[0], step[1])
        if P[1] <= med[1]:
            if med[0] > P[0]:
                large = med
            else:
                small = med
            med = P
        elif med[0] > P[0]:
            small = P
        else:
            large = P
        if math.isinf(small[1]):
            restore, btm = med, int(np.float32(med[0]) * r32)
            if btm == 0:
                want.append(None)
                continue
        elif large[0] - small[0] == 2:
            want.append(None)
            continue
        elif large[0] - med[0] >= med[0] - small[0]:
            nb = med[0] + int(math.floor((large[0] - med[0]) * 0.618 + 0.5))
            restore, btm = large, large[0] - nb
        else:
            nb = small[0] + int(math.floor((med[0] - small[0]) * 0.618 + 0.5))
            restore, btm = med, med[0] - nb
        want.append(restore[0] - btm)
    return want


def _check(steps, N):
    assert steps, "no steps"
    # the first step's B comes from the first merge at B = N
    assert steps[0][0] == N - int(np.float32(N) * np.float32(0.35))
    want = replay(steps, N)
    for k in range(len(steps) - 1):
        assert want[k] is not None, ("search ended early", k)
        assert steps[k + 1][0] == want[k], (k, steps[k + 1][0], want[k])
    assert want[-1] is None, "the run stopped while the search was still open"


CASES = [("LL", 1000, 11, 0), ("HH", 1000, 11, 1), ("LH", 2000, 16, 2), ("HL", 3000, 20, 3)]


@pytest.mark.parametrize("variant,N,B,seed", CASES)
def test_replay_matches_oracle_trace(orc, variant, N, B, seed):
    g = orc.dcsbm_variant(variant, N, B, seed=seed)
    _, steps = orc.partition_trace(g, seed=seed)
    _check(steps, N)


@pytest.mark.gpu
@pytest.mark.parametrize("variant,N,B,seed", CASES + [("HH", 20000, 32, 0)])
def test_engine_golden_section_follows_the_rule(sbp, capfd, variant, N, B, seed):
    g = graphs.dcsbm(variant, N, B, seed)
    capfd.readouterr()
    rep = sbp.partition(g, seed=seed, verbose=1)
    err = capfd.readouterr().err
    steps = [(int(m.group(1)), float(m.group(2)), int(m.group(3)))
             for m in re.finditer(r"\[sbp\] step \d+ B=(\d+) S=(\S+) itrs=(\d+)", err)]
    assert len(steps) == rep["outer_steps"]
    _check(steps, N)
    # the run ends at the bracket's middle point: the last step whose S was
    # at most every S before it
    med = None
    for st in steps:
        if med is None or st[1] <= med[1]:
            med = st
    assert rep["B"] == med[0] and rep["S"] == med[1]
