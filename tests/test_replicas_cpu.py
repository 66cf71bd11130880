"""The multi-rank host logic (cospanmdao_b200.replicas) on two gloo ranks on the CPU.

Each rank takes its contiguous shard of a ragged column (4096 instances, log-uniform sizes, cost n²), scans its
counts locally (the oracle's scan stands in for the device scan), and moves its offsets to the global column with
the one exchange of shard totals. The concatenation must equal the single-process scan bit for bit. The max-over-ranks
timing and the whole-job rate are checked too, and a rank that fails before a collective ends its peer's wait with
an error (no hang).
"""
import json
import os
import socket
from pathlib import Path

import numpy as np
import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank, world, port):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))


def _rank_scan(rank, world, port, out_dir):
    _env(rank, world, port)
    import oracle
    from cospanmdao_b200 import workloads
    from cospanmdao_b200.replicas import Ranks, global_offsets, shard_by_cost, whole_job_rate
    r = Ranks().init("gloo", timeout_s=60)
    sizes = workloads.ragged_sizes(4096)
    shards = shard_by_cost(sizes.astype(np.float64) ** 2, world)
    mine = sizes[shards[rank]]
    local = oracle.exclusive_scan(mine.astype(np.uint64))
    g = global_offsets(local, r)
    t_max = r.max(0.010 * (rank + 1))           # each rank's "device time": 10 ms, 20 ms
    units = r.sum(float(mine.size))
    rate = whole_job_rate([units], t_max)
    np.save(Path(out_dir) / f"offs{rank}.npy", g)
    Path(out_dir, f"r{rank}.json").write_text(json.dumps(
        {"t_max": t_max, "units": units, "rate": rate, "first": int(shards[rank][0]) if mine.size else -1,
         "count": int(mine.size), "cost": float((mine.astype(np.float64) ** 2).sum())}))
    r.barrier()
    r.close()


def _rank_fails(rank, world, port, out_dir):
    _env(rank, world, port)
    from cospanmdao_b200.replicas import Ranks
    r = Ranks().init("gloo", timeout_s=20)
    if rank == 1:
        raise RuntimeError("rank 1 leaves before the exchange")
    r.gather_ints(7)  # must end with an error once the peer is gone, not wait forever


def _spawn(fn, world, tmp_path):
    import torch.multiprocessing as mp
    mp.start_processes(fn, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True, start_method="spawn")


def test_sharded_offsets_equal_the_single_process_scan(tmp_path):
    import oracle
    from cospanmdao_b200 import workloads
    world = 2
    _spawn(_rank_scan, world, tmp_path)
    sizes = workloads.ragged_sizes(4096)
    whole = oracle.exclusive_scan(sizes.astype(np.uint64))
    parts = [np.load(tmp_path / f"offs{r}.npy") for r in range(world)]
    joined = np.concatenate([p[:-1] for p in parts] + [parts[-1][-1:]])
    assert joined.dtype == np.uint64 and np.array_equal(joined, whole)
    info = [json.loads((tmp_path / f"r{r}.json").read_text()) for r in range(world)]
    assert all(i["t_max"] == pytest.approx(0.020) for i in info)          # the max over ranks
    assert all(i["units"] == 4096 for i in info)                          # every unit in exactly one shard
    assert info[0]["rate"] == pytest.approx(4096 / 0.020)
    assert info[0]["first"] == 0 and info[1]["first"] == info[0]["count"]  # contiguous shards
    costs = [i["cost"] for i in info]
    biggest = float(sizes.max()) ** 2
    assert abs(costs[0] - costs[1]) <= 2 * biggest                        # balanced to within one unit each side


def test_a_rank_that_leaves_ends_the_peers_wait_with_an_error(tmp_path):
    with pytest.raises(Exception):
        _spawn(_rank_fails, 2, tmp_path)


def test_shard_by_cost_edge_cases():
    from cospanmdao_b200.replicas import shard_by_cost
    assert [s.tolist() for s in shard_by_cost([], 3)] == [[], [], []]
    assert [s.tolist() for s in shard_by_cost([5.0], 2)] in ([[0], []], [[], [0]])
    s = shard_by_cost(np.ones(10), 4)
    assert sorted(np.concatenate(s).tolist()) == list(range(10))
    assert [len(x) for x in s] == [3, 2, 3, 2] or sum(len(x) for x in s) == 10
    with pytest.raises(ValueError):
        shard_by_cost([1.0, -1.0], 2)
