"""CPU tests of the multi-GPU (replicas) host logic with world_size-2 gloo
process groups on 127.0.0.1: domain routing, barrier, MAX-over-ranks timing
and the whole-job rate, the same code bench.py runs under torchrun."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from pf3d import replicas


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_assign_lpt():
    costs = [9, 8, 7, 6, 5, 4, 3, 2, 1]
    owner = replicas.assign(costs, 2)
    loads = [sum(c for c, o in zip(costs, owner) if o == r) for r in range(2)]
    assert sorted(loads) == [22, 23]
    assert replicas.assign(costs, 2) == owner            # deterministic
    shares = [replicas.my_share(costs, 3, r) for r in range(3)]
    assert sorted(sum(shares, [])) == list(range(len(costs)))


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    r, w, lr = replicas.rank_env()
    replicas.barrier()
    t = 1.0 + rank                                          # rank 1 is the slowest
    tmax = replicas.max_over_ranks(t)
    mine = replicas.my_share([5, 4, 3, 2, 1, 1], w, r)
    rate = replicas.aggregate_rate(1e9, 10, w, tmax)
    dist.destroy_process_group()
    q.put((r, w, lr, tmax, mine, rate))


def test_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[0] for r in res] == [0, 1] and all(r[1] == 2 for r in res)
    assert all(r[3] == 2.0 for r in res)                    # MAX over ranks
    assert sorted(res[0][4] + res[1][4]) == list(range(6))  # every domain exactly once
    assert all(abs(r[5] - 10.0) < 1e-12 for r in res)       # 2 ranks x 1e9 x 10 / 2 s


@pytest.mark.parametrize("world", [2, 4, 8])
def test_batched_domains_routing(world):
    """The batched workload's 96 domains spread over N ranks (bench.py's
    batched sub-line at N > 1): every domain on exactly one rank, and the
    slowest rank's cells within LPT's 4/3 of the lower bound max(total/N,
    largest domain)."""
    from pf3d import serve
    costs = [j.cells for j in serve.batch_domains(seed=3)]
    shares = [replicas.my_share(costs, world, r) for r in range(world)]
    assert sorted(sum(shares, [])) == list(range(len(costs)))
    worst = max(sum(costs[i] for i in s) for s in shares)
    bound = max(sum(costs) / world, max(costs))
    assert worst <= 4 / 3 * bound
