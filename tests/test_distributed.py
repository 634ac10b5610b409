"""The multi-GPU plumbing on CPU: world_size-2 process groups over gloo.

Orbits shard across ranks with no data exchange in the integration; the
only collectives are the bench's reductions (MAX of device time, SUM of
work) and the sum of the potential-parameter gradient after the backward
pass (galpy_b200.adjoint.reduce_param_grad)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import sys

    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        from galpy_b200.adjoint import reduce_param_grad

        # bench aggregation: slowest rank's time, all ranks' work
        (ms,), (steps, nbad) = bench.over_ranks([10.0 + rank], [100.0 * (rank + 1), rank], dist,
                                                "cpu")
        # shards: distinct seeds, hence distinct orbits
        ics, _ = bench.workload(4, seed=bench.shard_seed(1, rank))
        gathered = [torch.zeros(4, 6, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(gathered, torch.from_numpy(ics))
        distinct = not torch.equal(gathered[0], gathered[1])
        # parameter gradient: summed over ranks; IC gradients stay local
        g = torch.full((7,), float(rank + 1), dtype=torch.float64)
        reduce_param_grad(g)
        q.put((rank, ms, steps, nbad, distinct, g.tolist()))
    finally:
        dist.destroy_process_group()


def test_two_rank_reductions_over_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, steps, nbad, distinct, g in out:
        assert ms == 11.0 and steps == 300.0 and nbad == 1.0
        assert distinct
        assert g == [3.0] * 7


def test_single_process_reductions_are_identity():
    import sys

    sys.path.insert(0, ROOT)
    import bench
    from galpy_b200.adjoint import reduce_param_grad

    assert bench.over_ranks([2.5], [7, 1], None, "cpu") == ([2.5], [7.0, 1.0])
    g = torch.ones(3, dtype=torch.float64)
    assert reduce_param_grad(g) is g and g.tolist() == [1.0] * 3
    with pytest.raises(Exception):
        bench.over_ranks([1.0], [1.0], object(), "cpu")
