"""The bench's N > 1 path on CPU: two gloo ranks, each timing its own
replica, agree on the slowest rank's time, and the whole-job rate counts
the units of every rank over that time (weak scaling, no data-path
collective)."""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    import bench
    r = bench.Ranks("gloo")
    assert (r.world, r.rank) == (world, rank)
    r.barrier()
    ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
    slowest = r.max(ms)
    out.put((rank, slowest, bench.whole_job_rate(1e9, r.world, slowest)))
    r.close()


def test_two_gloo_ranks_take_the_max_time():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(k, world, port, q)) for k in range(world)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in results] == [15.0, 15.0]
    # 2 ranks x 1e9 units in 15 ms = 133.33 G units/s
    assert abs(results[0][2] - 2e9 / 0.015 / 1e9) < 1e-9


def test_single_process_needs_no_process_group():
    import bench
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        os.environ.pop(k, None)
    r = bench.Ranks("gloo")
    assert r.world == 1 and r.dist is None and r.max(3.5) == 3.5
    r.close()
