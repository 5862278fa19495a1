"""Rank sharding of independent units (gvx.shard) on CPU: the partition is
cost-balanced and deterministic, and two gloo ranks that each compute only
their own units -- here with the oracle, the CPU restatement of the kernels --
assemble on rank 0 exactly the result of a single process computing all of
them.  Two workloads: per-list collision counts of uneven lists against one
map (C3's lists, scaled down) and squared distances at query voxels of
uneven EDT maps (C5's maps, scaled down)."""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "gpu-voxels_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _lists_case():
    from golden_cases import LIST_CASE, list_inputs
    bmap, ids, vox, offs = list_inputs(LIST_CASE)
    return bmap, ids, vox, offs


def _lists_compute(case, mine):
    import oracle
    bmap, ids, vox, offs = case
    out = []
    for k in mine:
        a, b = int(offs[k]), int(offs[k + 1])
        out.append(oracle.list_collide_map(ids[a:b], vox[a * 32:b * 32].copy(), bmap, 0, False))
    return torch.as_tensor(np.asarray(out, dtype=np.int64))


def _maps_case():
    rng = np.random.default_rng(3)
    scenes = []
    for i in range(7):
        dims = tuple(int(v) for v in rng.integers(8, 40, size=3))
        pts = (rng.random((int(rng.integers(5, 200)), 3)) * dims).astype(np.float32)
        q = rng.integers(0, int(np.prod(dims)), size=int(rng.integers(10, 50))).astype(np.uint32)
        scenes.append((dims, pts, q))
    return scenes


def _maps_compute(scenes, mine):
    import oracle
    out = []
    for k in mine:
        dims, pts, q = scenes[k]
        m = oracle.dvm_empty(dims)
        oracle.dvm_insert(m, dims, 1.0, pts)
        oracle.pba(m, dims)
        out.append(oracle.sqdist(m, dims, q).astype(np.int64))
    return torch.as_tensor(np.concatenate(out) if out else np.zeros(0, np.int64))


def _rank_main(rank: int, world: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank))
    from datetime import timedelta

    import torch.distributed as dist
    from gvx import shard

    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    try:
        lists = _lists_case()
        lengths = (lists[3][1:] - lists[3][:-1]).astype(np.float64)
        counts, mine_l, plan_l = shard.run_sharded(lengths, lambda m: _lists_compute(lists, m), lambda k: 1, dist)
        scenes = _maps_case()
        costs = [float(np.prod(s[0])) for s in scenes]
        sq, mine_m, plan_m = shard.run_sharded(costs, lambda m: _maps_compute(scenes, m),
                                               lambda k: scenes[k][2].shape[0], dist)
        out.put((rank, mine_l, mine_m, None if counts is None else counts.numpy(), None if sq is None else sq.numpy()))
    finally:
        dist.destroy_process_group()


def test_partition_is_balanced_and_deterministic():
    from gvx import shard
    rng = np.random.default_rng(0)
    costs = np.exp(rng.uniform(np.log(2e3), np.log(2e5), 4096))  # C3's list lengths
    for world in (1, 2, 4, 8):
        plan = shard.partition(costs, world)
        assert sorted(i for p in plan for i in p) == list(range(costs.shape[0]))
        assert plan == shard.partition(costs, world)
        assert shard.imbalance(costs, plan) < 1.01
    assert shard.partition([5.0, 1.0, 1.0, 1.0], 2) == [[0], [1, 2, 3]]
    assert shard.partition([3.0], 4) == [[0], [], [], []]


def test_two_gloo_ranks_assemble_the_single_process_result():
    from gvx import shard
    lists = _lists_case()
    lengths = (lists[3][1:] - lists[3][:-1]).astype(np.float64)
    want_counts, _, _ = shard.run_sharded(lengths, lambda m: _lists_compute(lists, m), lambda k: 1)
    scenes = _maps_case()
    want_sq, _, _ = shard.run_sharded([float(np.prod(s[0])) for s in scenes], lambda m: _maps_compute(scenes, m),
                                      lambda k: scenes[k][2].shape[0])
    assert int(want_counts.sum()) > 0

    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(k, world, port, q)) for k in range(world)]
    for p in procs:
        p.start()
    results = sorted((q.get(timeout=180) for _ in range(world)), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, l0, m0, counts, sq), (_, l1, m1, none_c, none_s) = results
    assert none_c is None and none_s is None  # only rank 0 receives the result
    assert sorted(l0 + l1) == list(range(lengths.shape[0])) and l0 and l1
    assert sorted(m0 + m1) == list(range(len(scenes))) and m0 and m1
    assert np.array_equal(counts, want_counts.numpy())
    assert np.array_equal(sq, want_sq.numpy())
