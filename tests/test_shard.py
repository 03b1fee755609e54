"""Sharding of independent solve units across ranks (host side, no GPU).

The units of a job -- (antenna, frequency, right-hand side) solves -- never
exchange data (the reference's sweep runs them independently,
apps/nec-cli/src/solve_session.rs:1794-1815), so a multi-GPU job is a
partition of the antennas plus a gather of the per-unit results on rank 0.
These tests run the partitioner on the uneven benchmark batch and the
gather as two gloo ranks on the host.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from nec_accel import shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_partition_every_unit_once_and_balanced():
    rng = np.random.default_rng(3)
    costs = rng.lognormal(10.0, 1.5, size=1000)
    for world in (1, 2, 3, 4, 8):
        parts = shard.partition(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        for p in parts:
            assert p == sorted(p)
        ld = shard.loads(costs, parts)
        # greedy largest-first: every rank within one unit's cost of the mean
        assert max(ld) - min(ld) <= costs.max() + 1e-6 * sum(ld)


def test_partition_edge_cases():
    assert shard.partition([], 3) == [[], [], []]
    assert shard.partition([5.0], 4) == [[0], [], [], []]
    # equal costs: round robin by rank, lower rank first
    assert shard.partition([1.0] * 5, 2) == [[0, 2, 4], [1, 3]]
    with pytest.raises(ValueError):
        shard.partition([1.0], 0)


def test_partition_uneven_benchmark_batch():
    import bench
    import nec_accel as acc

    wl = bench.uneven_workload(512)
    ants = [acc.Antenna(acc.wires_array(w), acc.sources_array(s), [f], g, None) for w, s, g, f in wl]
    sizes = [shard.antenna_sizes(a) for a in ants]
    assert all(n == sum(w[1] for w in wl[i][0]) for i, (n, *_rest) in enumerate(sizes))
    costs = [shard.unit_cost(*sz[:5], ground=sz[5]) for sz in sizes]
    parts = shard.partition_antennas(ants, 4)
    ld = shard.loads(costs, parts)
    assert sorted(i for p in parts for i in p) == list(range(len(ants)))
    assert max(ld) / min(ld) < 1.02


def _gather_worker(rank, world, port, n_total, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        costs = [float((i * 7919) % 97 + 1) for i in range(n_total)]
        parts = shard.partition(costs, world)
        mine = parts[rank]
        # per-unit results: a feedpoint row tagged with the job index
        local = [np.array([i, 1.0, 0.0, 2.0 * i, 0.5, 1e-3 * i, -1e-3 * i]) for i in mine]
        got = shard.gather_units(local, mine, n_total, dst=0)
        if rank == 0:
            ok = len(got) == n_total and all(int(r[0]) == i and r[3] == 2.0 * i for i, r in enumerate(got))
            q.put(("order", ok))
        else:
            q.put(("other", got is None))
        # a unit returned twice (rank 1 repeats its first index) is refused
        bad_idx = list(mine)
        if rank == 1 and bad_idx:
            bad_idx[-1] = parts[0][0]
        try:
            shard.gather_units(local, bad_idx, n_total, dst=0)
            q.put(("dup", rank != 0))
        except ValueError:
            q.put(("dup", rank == 0))
    finally:
        dist.destroy_process_group()


def test_gather_two_gloo_ranks_restores_job_order():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gather_worker, args=(r, 2, port, 53, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = [q.get(timeout=5) for _ in range(4)]
    assert all(ok for _, ok in res), res
    assert {k for k, _ in res} == {"order", "other", "dup"}
