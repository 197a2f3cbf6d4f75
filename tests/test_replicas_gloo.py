"""Multi-rank host logic on CPU: two gloo ranks agree on the matrix-to-rank
assignment without communicating, every matrix has exactly one owner, the
per-rank work is balanced, and the max-over-ranks timing / weak-scaling
throughput match the single-process formula."""
import os
import socket

import pytest
import torch.multiprocessing as mp

import replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, sizes, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        a = replicas.assign_to_ranks(sizes, world)
        mine = a[rank]
        my_ms = 10.0 + rank * 5.0  # rank 1 is the slow one
        mx = replicas.max_over_ranks(my_ms)
        tot = replicas.sum_over_ranks(sum(sizes[i] for i in mine))
        gathered = [None] * world
        dist.all_gather_object(gathered, a)
        q.put((rank, mine, mx, tot, gathered))
    finally:
        dist.destroy_process_group()


def test_two_rank_assignment_and_timing():
    sizes = [5, 900, 33, 33, 120, 7, 64, 640, 1, 250, 250, 19]
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, sizes, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    owned = sorted(i for _, mine, _, _, _ in res for i in mine)
    assert owned == list(range(len(sizes)))
    for _, _, mx, tot, gathered in res:
        assert mx == 15.0
        assert tot == sum(sizes)
        assert gathered[0] == gathered[1]  # both ranks computed the same map
    loads = [sum(sizes[i] for i in mine) for _, mine, _, _, _ in res]
    assert max(loads) - min(loads) <= max(sizes)


def test_weak_scaling_formula():
    assert replicas.weak_scaling_gbs(1e9, 10, 1000.0, 1) == pytest.approx(10.0)
    assert replicas.weak_scaling_gbs(1e9, 10, 1000.0, 4) == pytest.approx(40.0)
    a = replicas.assign_to_ranks([3, 3, 3], 1)
    assert a == [[0, 1, 2]]
    assert replicas.owner_of(replicas.assign_to_ranks([1, 2, 3, 4], 2)) == {3: 0, 0: 0, 2: 1, 1: 1}
