"""Batched and served partitioning (sbp_partition_batch, sbp_server_*).

The multi-job engine runs every job's kernels inside shared launches; a
job's virtual grid depends on its own sizes only, so each result must be the
same bits as the job partitioned alone: labels, B and MDL are compared for
equality, not within a tolerance."""
import numpy as np
import pytest

import graphs

pytestmark = pytest.mark.gpu


def _mix():
    gs = [graphs.dcsbm("LL", 1000, 11, 0), graphs.dcsbm("HH", 2000, 16, 1),
          graphs.dcsbm("LH", 5000, 24, 2), graphs.dcsbm("HL", 3000, 20, 3),
          graphs.hub_graph(N=6000, hub_in=5000, seed=4), graphs.weighted_graph(600, 5)]
    return gs, [11, 22, 33, 44, 55, 66]


@pytest.fixture(scope="module")
def solo(sbp):
    gs, seeds = _mix()
    out = []
    for g, s in zip(gs, seeds):
        rep = sbp.partition(g, seed=s)
        out.append((g.partitions.copy(), rep))
    return gs, seeds, out


def _same(lab, rep, lab0, rep0):
    assert rep["status"] == 0
    assert rep["B"] == rep0["B"]
    assert rep["S"] == rep0["S"]
    assert np.array_equal(lab, lab0)
    assert rep["nodal_itrs"] == rep0["nodal_itrs"]
    assert rep["accepted_moves"] == rep0["accepted_moves"]


def test_batch_matches_solo(sbp, solo):
    gs, seeds, ref = solo
    labs, reps, br = sbp.partition_batch(gs, seeds=seeds)
    assert br["count"] == len(gs) and br["max_active"] == len(gs)
    for i in range(len(gs)):
        _same(labs[i], reps[i], *ref[i])


def test_batch_budget_admits_in_order(sbp, solo):
    gs, seeds, ref = solo
    sizes = [sbp.job_bytes(g.N, g.E) for g in gs]
    budget = max(sizes) + min(sizes)  # the largest job never shares the device
    labs, reps, br = sbp.partition_batch(gs, seeds=seeds, hbm_budget=budget)
    assert br["peak_bytes"] <= budget
    assert br["max_active"] < len(gs)
    for i in range(len(gs)):
        _same(labs[i], reps[i], *ref[i])


def test_batch_job_over_budget(sbp, solo):
    gs, seeds, _ = solo
    small = min(sbp.job_bytes(g.N, g.E) for g in gs)
    with pytest.raises(sbp.SbpError, match="HBM budget"):
        sbp.partition_batch(gs, seeds=seeds, hbm_budget=small)


def test_batch_empty_and_one(sbp, solo):
    gs, seeds, ref = solo
    labs, reps, br = sbp.partition_batch([], seeds=[])
    assert labs == [] and br["count"] == 0
    labs, reps, _ = sbp.partition_batch(gs[:1], seeds=seeds[:1])
    _same(labs[0], reps[0], *ref[0])


def test_server_mix_equals_solo(sbp, solo):
    # requests arrive while others are on the device; each result is the
    # same as the job alone
    gs, seeds, ref = solo
    with sbp.Server() as srv:
        ids = [srv.submit(gs[i], seeds[i]) for i in range(3)]
        first = srv.poll(ids[0], timeout_ms=-1)
        ids += [srv.submit(gs[i], seeds[i]) for i in range(3, len(gs))]
        results = [first] + [srv.poll(j, timeout_ms=-1) for j in ids[1:]]
        st = srv.stats()
    assert st["submitted"] == len(gs) and st["completed"] == len(gs) and st["failed"] == 0
    for i, (lab, rep, times) in enumerate(results):
        _same(lab, rep, *ref[i])
        assert times["ms_latency"] >= times["ms_run"] >= 0.0
        assert times["ms_queue"] >= 0.0


def test_server_lanes_equal_solo(sbp, solo):
    # a low split spreads the requests over three lanes (engines on their
    # own streams and threads); every result is still the job alone
    gs, seeds, ref = solo
    with sbp.Server(lanes=3, lane_split=1500) as srv:
        ids = [srv.submit(g, s) for g, s in zip(gs, seeds)]
        res = [srv.poll(j, timeout_ms=-1) for j in ids]
        st = srv.stats()
    assert st["completed"] == len(gs) and st["failed"] == 0
    for i, (lab, rep, _) in enumerate(res):
        _same(lab, rep, *ref[i])


def test_server_submit_while_polling(sbp, solo):
    # a poll that waits while new requests arrive (the request table grows
    # under it) still returns the right job
    import threading
    import time
    gs, seeds, ref = solo
    with sbp.Server() as srv:
        ids = [None] * 40
        out = [None] * 40

        def collect():
            for i in range(40):
                while ids[i] is None:
                    time.sleep(0.0002)
                out[i] = srv.poll(ids[i], timeout_ms=-1)

        th = threading.Thread(target=collect)
        th.start()
        for i in range(40):
            k = i % len(gs)
            ids[i] = srv.submit(gs[k], seeds[k])
        th.join()
    for i in range(40):
        _same(out[i][0], out[i][1], *ref[i % len(gs)])


def test_server_one_at_a_time(sbp, solo):
    gs, seeds, ref = solo
    with sbp.Server(max_active=1, lanes=1) as srv:
        ids = [srv.submit(g, s) for g, s in zip(gs, seeds)]
        res = [srv.poll(j, timeout_ms=-1) for j in ids]
        assert srv.stats()["max_active_seen"] == 1
    for i, (lab, rep, _) in enumerate(res):
        _same(lab, rep, *ref[i])


def test_server_errors(sbp, solo):
    gs, seeds, _ = solo
    sizes = [sbp.job_bytes(g.N, g.E) for g in gs]
    i0, i1 = int(np.argmin(sizes)), int(np.argmax(sizes))
    with sbp.Server(hbm_budget=sizes[i0]) as srv:
        with pytest.raises(sbp.SbpError, match="HBM budget"):
            srv.submit(gs[i1], 0)
        j = srv.submit(gs[i0], seeds[i0])
        assert srv.poll(j, timeout_ms=-1) is not None
        with pytest.raises(sbp.SbpError, match="unknown request"):
            srv.poll(j, timeout_ms=0)


def test_graph_replay_same_bits(sbp, solo):
    # ticks of queued sweeps captured as CUDA graphs and replayed (the
    # default) give the same partition as direct launches, alone and in a
    # batch
    gs, seeds, ref = solo
    for i in (0, 2, 4):
        assert ref[i][1]["graph_captures"] > 0 and ref[i][1]["graph_replays"] > 0
        rep = sbp.partition(gs[i], seed=seeds[i], use_graphs=0)
        assert rep["graph_captures"] == 0 and rep["graph_replays"] == 0
        _same(gs[i].partitions, rep, *ref[i])
    labs, reps, _ = sbp.partition_batch(gs, seeds=seeds, use_graphs=0)
    for i in range(len(gs)):
        _same(labs[i], reps[i], *ref[i])


def test_server_two_pollers_one_request(sbp, solo):
    # two threads wait on the same request: one collects it, the other is
    # told it is gone (never a freed request)
    import threading
    gs, seeds, ref = solo
    i = int(np.argmax([g.N for g in gs]))
    with sbp.Server() as srv:
        for _ in range(3):
            j = srv.submit(gs[i], seeds[i])
            got, errs = [], []

            def poll():
                try:
                    got.append(srv.poll(j, timeout_ms=-1))
                except sbp.SbpError as e:
                    errs.append(str(e))

            ths = [threading.Thread(target=poll) for _ in range(2)]
            for t in ths:
                t.start()
            for t in ths:
                t.join(timeout=120)
            assert not any(t.is_alive() for t in ths)
            assert len(got) == 1 and len(errs) == 1, (got, errs)
            assert "collected" in errs[0] or "unknown request" in errs[0]
            _same(got[0][0], got[0][1], *ref[i])
