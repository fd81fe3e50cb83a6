"""The multi-rank paths on CPU, two ``gloo`` ranks on 127.0.0.1 with fake solves standing
in for the device solves (which need a GPU): independent problems sharded by cost and
gathered; one objective split over the ranks (the tPhys broadcast and the all-reduce of
gradient and stage compliances); the max-over-ranks timing reduction.  No GPU."""

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def test_partition_balances_and_covers(pkg):
    from sttopt_b200 import sharding

    costs = [5, 1, 9, 3, 3, 7, 2, 8]
    parts = sharding.partition(costs, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)
    assert sharding.partition(costs, 3) == parts  # deterministic
    assert sharding.partition([], 2) == [[], []]
    assert sharding.partition([4.0], 3) == [[0], [], []]
    with pytest.raises(ValueError):
        sharding.partition(costs, 0)
    assert len({sharding.rank_seed(3, r) for r in range(8)}) == 8


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _fake_solve(xs, ws, ns, scale=1.0):
    # stands in for the device solve: objective sum(x w) * n, gradient w * n
    return [dict(objective=(x * w).sum() * n * scale, gradient=w * n * scale) for x, w, n in zip(xs, ws, ns)]


def _worker(rank, world, port, result_q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    from __graft_entry__ import load_package

    load_package()
    from sttopt_b200 import sharding

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        g = torch.Generator().manual_seed(11)
        sizes = [(8, 4), (16, 8), (12, 6), (8, 4), (24, 12), (16, 8), (8, 4)]
        xs = [torch.rand(ny, nx, generator=g, dtype=torch.float64) for nx, ny in sizes]
        ws = [torch.rand(ny, nx, generator=g, dtype=torch.float64) for nx, ny in sizes]
        ns = [4, 16, 8, 5, 12, 7, 9]
        idx, outs = sharding.objective_and_gradient_sharded(xs, ws, ns, solve=_fake_solve, scale=2.0)
        grads = sharding.gather(idx, [o["gradient"] for o in outs], len(xs))
        objs = sharding.gather(idx, [o["objective"].reshape(1) for o in outs], len(xs))
        t = sharding.max_over_ranks(float(rank + 1) * 1.5)
        ok = all(torch.equal(grads[i], ws[i] * ns[i] * 2.0) for i in range(len(xs)))
        ok = ok and all(torch.allclose(objs[i][0], (xs[i] * ws[i]).sum() * ns[i] * 2.0) for i in range(len(xs)))
        result_q.put((rank, sorted(idx), ok, t))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_gather(pkg):
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=5) for _ in range(world))
    shares = [r[1] for r in res]
    assert sorted(i for s in shares for i in s) == list(range(7))  # every unit once
    assert all(r[2] for r in res)                                  # gathered results exact
    assert all(r[3] == 3.0 for r in res)                           # max over ranks


def test_stage_partition(pkg):
    from sttopt_b200 import sharding

    for n_stage, world in [(16, 1), (16, 2), (16, 3), (16, 8), (4, 8), (17, 4)]:
        parts = sharding.stage_partition(n_stage, world)
        assert sorted(s for p in parts for s in p) == list(range(n_stage))
        assert all(p == sorted(p) for p in parts)
        loads = [len(p) + (1.0 if r == 0 else 0.0) for r, p in enumerate(parts)]
        assert max(loads) - min(loads) <= 1.0
    assert len(sharding.stage_partition(16, 2, heat_cost=0.0)[0]) == 8
    with pytest.raises(ValueError):
        sharding.stage_partition(4, 0)


def _fake_part(x, w, *, n_stage, stages, tphys, publish, calls=None):
    # stands in for the device share: tPhys from x (owner only, published at once), a
    # compliance and a gradient term per stage, the heat adjoint's term on the owner
    if tphys is None:
        tPhys = (x * x + 0.25) / (x * x + 0.25).max()
        if publish is not None:
            publish(tPhys)
    else:
        tPhys = tphys
    m = [(tPhys <= (s + 1) / n_stage).to(x.dtype) for s in stages]
    c_s = torch.stack([(x * mk).sum() * (s + 1) for s, mk in zip(stages, m)]) if stages else x.new_zeros(0)
    grad = sum(((s + 1) * mk for s, mk in zip(stages, m)), torch.zeros_like(x))
    if tphys is None:
        grad = grad + 0.5 * w
    return dict(c_s=c_s, gradient=grad, tPhys=tPhys)


def _split_worker(rank, world, port, result_q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    from __graft_entry__ import load_package

    load_package()
    from sttopt_b200 import sharding

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        g = torch.Generator().manual_seed(5)
        x = torch.rand(6, 10, generator=g, dtype=torch.float64)
        w = torch.rand(6, 10, generator=g, dtype=torch.float64) - 0.5
        out = sharding.objective_and_gradient_split(x, w, n_stage=16, solve=_fake_part)
        # the whole objective on one rank, the reference result
        full = _fake_part(x, w, n_stage=16, stages=list(range(16)), tphys=None, publish=None)
        J_t = (w * full["tPhys"]).sum()
        ok = (torch.allclose(out["c_s"], full["c_s"], rtol=1e-15, atol=0)
              and torch.allclose(out["gradient"], full["gradient"], rtol=1e-15, atol=1e-15)
              and torch.equal(out["tPhys"], full["tPhys"])
              and torch.allclose(out["objective"], full["c_s"].sum() + J_t, rtol=1e-15, atol=0))
        result_q.put((rank, out["stages"], bool(ok)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_one_objective(pkg):
    """One objective's stages over two gloo ranks: rank 0 solves the heat field and
    broadcasts tPhys, each rank its stages, one all-reduce combines gradient and stage
    compliances; every rank ends with the one-rank result."""
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_split_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=5) for _ in range(world))
    assert sorted(s for r in res for s in r[1]) == list(range(16))  # every stage once
    assert len(res[0][1]) <= len(res[1][1])                          # rank 0 also carries the heat work
    assert all(r[2] for r in res)
