"""CPU tests of the multi-GPU batch dispatcher's host logic: two gloo ranks
(processes) shard a batch, each "reduces" its share through a stand-in for
the single-GPU batch call, and rank 0 gathers every complex's result in input
order.  The stand-in is the oracle (checker only); no GPU is used."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from specseqplusplus_b200.multi import shard


def test_shard_balances_and_covers():
    ncols = [100, 5, 5, 80, 40, 40, 3, 7, 60]
    parts = shard(ncols, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(ncols)))
    loads = [sum(ncols[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(ncols)
    assert shard(ncols, 3) == parts  # every rank computes the same assignment
    assert shard([], 2) == [[], []]
    assert shard([4], 3) == [[0], [], []]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_batch(mats, params, device):
    import oracle

    out = []
    for m in mats:
        r = oracle.reduce(m)
        out.append((r.pairs, r.essential))
    return out


def _worker(rank, world, port, q):
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.dirname(here))
    sys.path.insert(0, os.path.join(os.path.dirname(here), "oracle"))
    import datetime

    import torch.distributed as dist

    from specseqplusplus_b200 import Params, workloads
    from specseqplusplus_b200.multi import reduce_batch

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mats, _ = workloads.batch_of_rips(9, seed=31, n_min=60, n_max=400, threads=1)
        res = reduce_batch(mats, Params(), reduce_fn=_oracle_batch)
        if rank == 0:
            import oracle

            ok = len(res) == len(mats) and all(
                np.array_equal(p, oracle.reduce(m).pairs) and np.array_equal(e, oracle.reduce(m).essential)
                for (p, e), m in zip(res, mats))
            q.put(("ok" if ok else "mismatch", len(res)))
        else:
            q.put(("none" if res is None else "unexpected", 0))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_gather_in_input_order():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got == [("none", 0), ("ok", 9)]


def _oracle_built(reqs, params, device):
    import oracle

    from specseqplusplus_b200 import gen

    out = []
    for req in reqs:
        m = gen.rips_from_points(req[1], req[2], req[3]) if req[0] == "rips" else gen.lowerstar_from_field(req[1], req[2])
        r = oracle.reduce(m)
        out.append((r.pairs, r.essential))
    return out


def _requests():
    from specseqplusplus_b200 import gen

    reqs = []
    for i in range(7):
        if i % 3 == 2:
            reqs.append(("lowerstar", gen.field(5 + i, 1.0, i), 3))
        else:
            reqs.append(("rips", gen.points(60 + 40 * i, 2 + i % 2, i), 0.2, 2 + i % 2))
    return reqs


def _worker_built(rank, world, port, q):
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.dirname(here))
    sys.path.insert(0, os.path.join(os.path.dirname(here), "oracle"))
    import datetime

    import torch.distributed as dist

    from specseqplusplus_b200 import Params
    from specseqplusplus_b200.multi import reduce_requests

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        reqs = _requests()
        res = reduce_requests(reqs, Params(), reduce_fn=_oracle_built)
        if rank == 0:
            want = _oracle_built(reqs, None, 0)
            ok = len(res) == len(reqs) and all(np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
                                               for a, b in zip(res, want))
            q.put(("ok" if ok else "mismatch", len(res)))
        else:
            q.put(("none" if res is None else "unexpected", 0))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_point_cloud_and_field_requests():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker_built, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got == [("none", 0), ("ok", 7)]
