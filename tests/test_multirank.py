"""Replica sharding across ranks (one process per GPU in production), run here
as world-size-2 gloo process groups on the CPU: the whole-job aggregation of
bench.py and the per-rank workload seeds."""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as tmp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    conv = [100, 37][rank]
    t = [2.0, 3.5][rank]
    e2e = [10.0, 7.0][rank]
    r = bench.aggregate_ranks(conv, t, e2e, dist, "cpu")
    r_none = bench.aggregate_ranks(conv, t, None, dist, "cpu")
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, r, r_none))


def test_aggregate_ranks_gloo_world2():
    ctx = tmp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = [q.get(timeout=120) for _ in ps]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, r, r_none in res:
        assert r == (137.0, 3.5, 17.0)            # summed systems, max time, summed e2e
        assert r_none == (137.0, 3.5, None)


def test_single_rank_passthrough():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.aggregate_ranks(5, 1.5, None, None, "cpu") == (5.0, 1.5, None)


def test_rank_workloads_are_disjoint():
    sys.path.insert(0, ROOT)
    from firecore_b200 import systems as S
    a = S.config_replicas(seed=1, nrep=4)
    b = S.config_replicas(seed=1 + 7919, nrep=4)
    assert not np.allclose(a.pos, b.pos)


def _workload_worker(rank, world, port, out):
    """Each rank builds its own share exactly as bench.py does (generator only,
    host side) and the ranks compare fingerprints through the process group."""
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    from firecore_b200 import systems as S
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    fps = []
    for kind in ("replicas", "uneven"):
        _, b = bench.workload(rank, 32, kind)
        fps.append(float(np.abs(b.pos).sum()))
    prod = S.config_uneven(seed=2002 + 7919 * rank, nsys=32)       # the learned workload's production share
    train = S.config_uneven(seed=1001 + 7919 * rank, nsys=32)      # and its training share
    fps += [float(np.abs(prod.pos).sum()), float(np.abs(train.pos).sum())]
    mine = torch.tensor(fps, dtype=torch.float64)
    allfp = [torch.zeros_like(mine) for _ in range(world)]
    dist.all_gather(allfp, mine)
    again = [float(np.abs(bench.workload(rank, 32, "uneven")[1].pos).sum())]
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, [t.tolist() for t in allfp], fps, again))


def test_rank_shares_are_disjoint_and_reproducible_gloo_world2():
    ctx = tmp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_workload_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = [q.get(timeout=300) for _ in ps]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, allfp, fps, again in res:
        assert allfp[rank] == fps
        # every workload differs between the two ranks
        assert all(abs(a - b) > 1e-6 * abs(a) for a, b in zip(allfp[0], allfp[1]))
        # and a rank regenerates the same share
        assert again[0] == fps[1]
