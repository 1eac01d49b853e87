"""Sharding of the batched workload over ranks (the multi-GPU path of bench.py):
the cost-model bin-pack, and two gloo ranks on the CPU that must agree on the
assignment, cover every instance exactly once and reduce the job time as the
maximum over ranks (the same steps bench.py takes over NCCL)."""
import os
import socket

import numpy as np
import pytest

from v2rdm_casscf_b200.shard import instance_cost, partition


def test_partition_is_complete_disjoint_and_balanced():
    rng = np.random.default_rng(0)
    for world in (1, 2, 3, 8):
        costs = list(rng.uniform(0.1, 10.0, 97))
        parts = partition(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(97))
        assert parts == partition(costs, world)  # deterministic
        loads = [sum(costs[i] for i in p) for p in parts]
        # longest-first greedy: no rank exceeds the mean by more than one instance
        assert max(loads) <= sum(costs) / world + max(costs) + 1e-9


def test_cost_model_grows_with_size():
    from v2rdm_casscf_b200 import V2RDMSolver

    c = []
    for n in (8, 12, 16):
        s = V2RDMSolver([n], n // 2, n // 2)
        c.append(instance_cost(s.dimx, s.nconstraints, s.dimensions))
    assert c[0] < c[1] < c[2]


def _rank(rank, world, port, out):
    import torch
    import torch.distributed as dist

    from v2rdm_casscf_b200.hamiltonian import batch_sizes, synthetic
    from v2rdm_casscf_b200.shard import workload_costs

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        spaces = [synthetic(int(n), s) for s, n in enumerate(batch_sizes(24))]
        parts = partition(workload_costs(spaces), world)
        mine = parts[rank]
        got = [None] * world
        dist.all_gather_object(got, mine)
        t = torch.tensor([float(len(mine)) + 0.5 * rank], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        # stub per-instance results, gathered the way bench.py gathers the solves'
        from v2rdm_casscf_b200.shard import gather_results

        stub = [dict(e_total=-1.5 * i, status=0 if i % 5 else -3, oiter=100 + i) for i in mine]
        allres = gather_results(mine, stub, world, dist)
        out.put((rank, parts, got, float(t[0]), allres))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_and_cover_everything():
    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort(key=lambda r: r[0])
    (_, parts0, got0, m0, all0), (_, parts1, got1, m1, all1) = res
    assert parts0 == parts1 == got0 == got1
    assert sorted(parts0[0] + parts0[1]) == list(range(24))
    assert m0 == m1 == max(len(parts0[0]), len(parts0[1]) + 0.5)
    # every instance's result reached both ranks, in instance order
    assert all0 == all1 == [(i, -1.5 * i, 0 if i % 5 else -3, 100 + i) for i in range(24)]
