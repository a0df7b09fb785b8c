"""The multi-rank plumbing of bench.py on CPU: two gloo ranks (one process
each, as torchrun starts them) take the barrier and agree on the max over
ranks; the reference arm runs on rank 0 alone."""
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

RANK_SCRIPT = r"""
import sys
sys.path.insert(0, {root!r})
import bench
rank, world, local = bench.dist_env()
d = bench.Dist(world, local, backend="gloo")
d.barrier()
m = d.max(10.0 * (rank + 1))
d.barrier()
d.close()
print("rank", rank, "max", m)
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run_ranks(code, world=2, extra=()):
    port = _free_port()
    procs = []
    for rank in range(world):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, *code, *extra], env=env, cwd=ROOT,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    out = []
    for p in procs:
        o, e = p.communicate(timeout=300)
        out.append((p.returncode, o, e))
    return out


def test_two_gloo_ranks_barrier_and_max():
    res = _run_ranks(["-c", RANK_SCRIPT.format(root=ROOT)])
    for rank, (rc, o, e) in enumerate(res):
        assert rc == 0, e[-2000:]
        assert f"rank {rank} max 20.0" in o


def test_reference_arm_runs_on_rank_zero_only():
    # rank 1 of the reference arm exits 0 without work and prints nothing
    res = _run_ranks(["bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1",
                      "--warmup", "1"])
    rc, o, e = res[1]
    assert rc == 0, e[-2000:]
    assert o.strip() == ""


def test_phase_rates():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    tot = {"bytes_nodal": 2e9, "bytes_rebuild": 1e9, "bytes_merge": 5e8, "ms_nodal": 100.0,
           "ms_rebuild": 50.0, "ms_merge": 0.0}
    r = bench.phase_rates(tot, 250.0, 2)
    assert abs(r["nodal"] - 20.0) < 1e-12 and abs(r["rebuild"] - 20.0) < 1e-12
    assert r["merge"] is None
    assert abs(r["end_to_end"] - 14.0) < 1e-12 and r["bytes_per_step"] == 1.75e9


SHARD_SCRIPT = r"""
import json, sys
sys.path.insert(0, {root!r})
import numpy as np
import bench
from gsap_b200.shard import gather_results, shard_jobs
rank, world, local = bench.dist_env()
d = bench.Dist(world, local, backend="gloo")
costs = [int(c) for c in np.random.default_rng(0).integers(1000, 50000, 37)]
mine = shard_jobs(costs, world)[rank]
# each rank's stand-in for its partition_batch share
labels = [np.arange(10 + i, dtype=np.int32) % (i + 2) for i in mine]
reports = [{{"job": i, "rank": rank, "B": i + 2}} for i in mine]
tot = d.sum(len(mine))
labs, reps = gather_results(mine, labels, reports, world, rank)
d.barrier()
d.close()
if rank == 0:
    ok = all(np.array_equal(labs[i], np.arange(10 + i) % (i + 2)) and reps[i]["job"] == i
             for i in range(len(costs)))
    print(json.dumps({{"n": len(labs), "ok": ok, "tot": tot,
                      "ranks": sorted(set(r["rank"] for r in reps))}}))
else:
    print(json.dumps({{"none": labs is None and reps is None}}))
"""


def test_shard_jobs_covers_and_balances():
    import sys
    sys.path.insert(0, ROOT)
    from gsap_b200.shard import shard_jobs
    costs = [50, 10, 40, 30, 30, 20, 5, 5]
    for world in (1, 2, 3, 8, 10):
        plan = shard_jobs(costs, world)
        assert len(plan) == world
        flat = sorted(i for p in plan for i in p)
        assert flat == list(range(len(costs)))
        assert all(p == sorted(p) for p in plan)
        loads = [sum(costs[i] for i in p) for p in plan]
        if world <= len(costs):
            # greedy longest-first: no rank exceeds the lightest by more than one job
            assert max(loads) - min(loads) <= max(costs)


def test_two_gloo_ranks_shard_and_gather():
    import json
    res = _run_ranks(["-c", SHARD_SCRIPT.format(root=ROOT)])
    for rc, o, e in res:
        assert rc == 0, e[-2000:]
    r0 = json.loads(res[0][1].strip().splitlines()[-1])
    r1 = json.loads(res[1][1].strip().splitlines()[-1])
    assert r0 == {"n": 37, "ok": True, "tot": 37.0, "ranks": [0, 1]}
    assert r1 == {"none": True}
